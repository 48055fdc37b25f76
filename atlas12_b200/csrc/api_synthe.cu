// api_synthe.cu -- C ABI: context management and the SYNTHE entry points.
#include <cmath>
#include <cstdlib>

#include "api_common.cuh"
#include "synthe.cuh"
#include "synthe_h.cuh"

using namespace atlasgpu;

extern "C" {

int atlasgpu_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int atlasgpu_create(atlasgpu_ctx** out, const atlasgpu_opts* opts) {
  if (!out) return ATLASGPU_EINVAL;
  *out = nullptr;
  atlasgpu_ctx* ctx = new atlasgpu_ctx();
  if (opts) {
    ctx->device = opts->device;
    ctx->precision = opts->precision;
    ctx->stream = (cudaStream_t)opts->stream;
  }
  if (ctx->precision != ATLASGPU_PREC_FP64 && ctx->precision != ATLASGPU_PREC_MIXED) {
    delete ctx;
    return ATLASGPU_EINVAL;
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return ATLASGPU_ECUDA;
  }
  if (!ctx->stream) {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      delete ctx;
      return ATLASGPU_ECUDA;
    }
    ctx->own_stream = true;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, ctx->device) == cudaSuccess) {
    ctx->nsm = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
  }
  if (cudaMalloc(&ctx->ops, sizeof(JoshOps)) != cudaSuccess) {
    cudaGetLastError();
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ATLASGPU_ENOMEM;
  }
  *out = ctx;
  return ATLASGPU_OK;
}

int atlasgpu_destroy(atlasgpu_ctx* ctx) {
  if (!ctx) return ATLASGPU_EINVAL;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->bufs) cudaFree(kv.second.first);
  if (ctx->ops) cudaFree(ctx->ops);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return ATLASGPU_OK;
}

const char* atlasgpu_last_error(atlasgpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int atlasgpu_set_precision(atlasgpu_ctx* ctx, int precision) {
  if (!ctx) return ATLASGPU_EINVAL;
  if (precision != ATLASGPU_PREC_FP64 && precision != ATLASGPU_PREC_MIXED)
    return fail(ctx, ATLASGPU_EINVAL, "precision %d", precision);
  ctx->precision = precision;
  return ATLASGPU_OK;
}

int atlasgpu_set_stream(atlasgpu_ctx* ctx, void* stream) {
  if (!ctx) return ATLASGPU_EINVAL;
  cudaSetDevice(ctx->device);
  if (ctx->own_stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    ctx->own_stream = false;
  }
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
  } else {
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  return ATLASGPU_OK;
}

int atlasgpu_synchronize(atlasgpu_ctx* ctx) {
  if (!ctx) return ATLASGPU_EINVAL;
  CK(cudaStreamSynchronize(ctx->stream));
  return ATLASGPU_OK;
}

int64_t atlasgpu_launch_count(atlasgpu_ctx* ctx) { return ctx ? ctx->launches : -1; }

int atlasgpu_enable_timing(atlasgpu_ctx* ctx, int on) {
  if (!ctx) return ATLASGPU_EINVAL;
  ctx->timing = on != 0;
  return ATLASGPU_OK;
}

double atlasgpu_kernel_ms(atlasgpu_ctx* ctx, const char* name) {
  if (!ctx || !name) return -1.0;
  auto it = ctx->kms.find(name);
  return it == ctx->kms.end() ? -1.0 : it->second;
}

double atlasgpu_kernel_work(atlasgpu_ctx* ctx, const char* name) {
  if (!ctx || !name) return -1.0;
  auto it = ctx->kwork.find(name);
  return it == ctx->kwork.end() ? -1.0 : it->second;
}

int atlasgpu_set_operators(atlasgpu_ctx* ctx, const double* xtau8, const double* coefj,
                           const double* coefh, const double* ch_j, const double* ck_j) {
  if (!ctx || !xtau8 || !coefj || !coefh || !ch_j || !ck_j)
    return fail(ctx, ATLASGPU_EINVAL, "set_operators: null argument");
  if (!finite_all(xtau8, kNx) || !finite_all(coefj, kNx * kNx) || !finite_all(coefh, kNx * kNx) ||
      !finite_all(ch_j, kNx) || !finite_all(ck_j, kNx))
    return fail(ctx, ATLASGPU_ENONFINITE, "set_operators: non-finite operator entry");
  for (int i = 1; i < kNx; ++i)
    if (!(xtau8[i] > xtau8[i - 1])) return fail(ctx, ATLASGPU_EINVAL, "XTAU8 not increasing");
  JoshOps h;
  memcpy(h.xtau, xtau8, sizeof h.xtau);
  memcpy(h.ch, ch_j, sizeof h.ch);
  memcpy(h.ck, ck_j, sizeof h.ck);
  memcpy(h.coefj, coefj, sizeof h.coefj);
  memcpy(h.coefh, coefh, sizeof h.coefh);
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(ctx->ops, &h, sizeof h, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->ops_set = true;
  return ATLASGPU_OK;
}

// ---------------------------------------------------------------- grid/bin
int atlasgpu_synthe_grid(double wlbeg, double wlend, double resolu, atlasgpu_grid* g) {
  if (!g || !(wlbeg > 0.0) || !(wlend > wlbeg) || !(resolu > 0.0)) return ATLASGPU_EINVAL;
  g->ratio = 1.0 + 1.0 / resolu;
  g->ratiolg = log(g->ratio);
  g->length = (int32_t)(log(wlend / wlbeg) / g->ratiolg);
  g->ixwlbeg = (int32_t)(log(wlbeg) / g->ratiolg);
  g->wbegin = exp((double)g->ixwlbeg * g->ratiolg);
  if (g->wbegin < wlbeg) {
    g->ixwlbeg = g->ixwlbeg + 1;
    g->wbegin = exp((double)g->ixwlbeg * g->ratiolg);
  }
  return ATLASGPU_OK;
}

static int bin_core(atlasgpu_ctx* ctx, const double* d_wl, int64_t n, double ratiolg,
                    int32_t ixwlbeg, int32_t* d_nb, int64_t* flagged_host, int64_t cap,
                    int64_t* nflag_out) {
  unsigned long long* d_nf;
  int64_t* d_fl;
  int r;
  if ((r = bufT(ctx, "bin_nflag", 1, &d_nf))) return r;
  if ((r = bufT(ctx, "bin_flag", (size_t)cap, &d_fl))) return r;
  CK(cudaMemsetAsync(d_nf, 0, sizeof(unsigned long long), ctx->stream));
  {
    Timer tm(ctx, "synthe_bin");
    k_bin<<<grid_for(ctx, n, 256, 16), 256, 0, ctx->stream>>>(d_wl, n, ratiolg, ixwlbeg, d_nb,
                                                               d_fl, d_nf, cap);
    CKL(ctx);
  }
  unsigned long long nf = 0;
  CK(cudaMemcpyAsync(&nf, d_nf, sizeof nf, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if ((int64_t)nf > cap) return fail(ctx, ATLASGPU_EINVAL, "bin: %llu boundary cases exceed %lld", nf, (long long)cap);
  if (flagged_host && nf) CK(cudaMemcpy(flagged_host, d_fl, nf * sizeof(int64_t), cudaMemcpyDeviceToHost));
  *nflag_out = (int64_t)nf;
  return 0;
}

int atlasgpu_synthe_bin_dev(atlasgpu_ctx* ctx, const double* d_wlvac, int64_t n, double ratiolg,
                            int32_t ixwlbeg, int32_t* d_nbuff, int64_t* n_flagged) {
  if (!ctx || n < 0 || (n > 0 && (!d_wlvac || !d_nbuff)) || !(ratiolg > 0.0))
    return fail(ctx, ATLASGPU_EINVAL, "synthe_bin_dev: bad argument");
  if (n == 0) {
    if (n_flagged) *n_flagged = 0;
    return 0;
  }
  cudaSetDevice(ctx->device);
  const int64_t cap = 1 << 20;
  std::vector<int64_t> fl(cap);
  int64_t nf = 0;
  int r = bin_core(ctx, d_wlvac, n, ratiolg, ixwlbeg, d_nbuff, fl.data(), cap, &nf);
  if (r) return r;
  // boundary cases: the host C library log decides (bit-exact with the reader)
  for (int64_t k = 0; k < nf; ++k) {
    double w;
    CK(cudaMemcpy(&w, d_wlvac + fl[k], sizeof w, cudaMemcpyDeviceToHost));
    const int32_t nb = (int32_t)(log(w) / ratiolg + 0.5) - ixwlbeg + 1;
    CK(cudaMemcpy(d_nbuff + fl[k], &nb, sizeof nb, cudaMemcpyHostToDevice));
  }
  if (n_flagged) *n_flagged = nf;
  return 0;
}

int atlasgpu_synthe_bin(atlasgpu_ctx* ctx, const double* wlvac, int64_t n, double ratiolg,
                        int32_t ixwlbeg, int32_t* nbuff_out) {
  if (!ctx || n < 0 || (n > 0 && (!wlvac || !nbuff_out)) || !(ratiolg > 0.0))
    return fail(ctx, ATLASGPU_EINVAL, "synthe_bin: bad argument");
  if (n == 0) return 0;
  cudaSetDevice(ctx->device);
  double* d_wl;
  int32_t* d_nb;
  int r;
  if ((r = bufT(ctx, "bin_wl", (size_t)n, &d_wl)) || (r = bufT(ctx, "bin_nb", (size_t)n, &d_nb))) return r;
  CK(cudaMemcpyAsync(d_wl, wlvac, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  const int64_t cap = 1 << 20;
  std::vector<int64_t> fl(cap);
  int64_t nf = 0;
  if ((r = bin_core(ctx, d_wl, n, ratiolg, ixwlbeg, d_nb, fl.data(), cap, &nf))) return r;
  CK(cudaMemcpy(nbuff_out, d_nb, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  for (int64_t k = 0; k < nf; ++k)
    nbuff_out[fl[k]] = (int32_t)(log(wlvac[fl[k]]) / ratiolg + 0.5) - ixwlbeg + 1;
  return 0;
}

// ---------------------------------------------------------------- continuum
int atlasgpu_synthe_continuum(atlasgpu_ctx* ctx, const double* wledge, int nedge,
                              const double* continall, int stride, int nrhox, double wbegin,
                              double ratio, int length, float* continuum_out) {
  if (!ctx || !wledge || !continall || !continuum_out || nedge < 2 || nrhox < 1 ||
      nrhox > kKwMax || length < 1 || stride < 3 * (nedge - 1))
    return fail(ctx, ATLASGPU_EINVAL, "synthe_continuum: bad argument");
  for (int i = 1; i < nedge; ++i)
    if (!(wledge[i] > wledge[i - 1])) return fail(ctx, ATLASGPU_EINVAL, "wledge not increasing");
  if (!finite_all(continall, (size_t)nrhox * stride))
    return fail(ctx, ATLASGPU_ENONFINITE, "synthe_continuum: non-finite table entry");
  cudaSetDevice(ctx->device);
  double *d_we, *d_ca;
  float* d_out;
  int r;
  if ((r = bufT(ctx, "cont_we", nedge, &d_we)) || (r = bufT(ctx, "cont_ca", (size_t)nrhox * stride, &d_ca)) ||
      (r = bufT(ctx, "cont_out", (size_t)nrhox * length, &d_out)))
    return r;
  CK(cudaMemcpyAsync(d_we, wledge, nedge * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_ca, continall, (size_t)nrhox * stride * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  {
    Timer tm(ctx, "synthe_continuum");
    dim3 g((length + 255) / 256 < 4096 ? (length + 255) / 256 : 4096, nrhox);
    k_continuum<<<g, 256, 0, ctx->stream>>>(d_we, nedge, d_ca, stride, nrhox, wbegin, ratio, length, d_out);
    CKL(ctx);
  }
  CK(cudaMemcpyAsync(continuum_out, d_out, (size_t)nrhox * length * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

// ---------------------------------------------------------------- line opacity
int atlasgpu_synthe_line_opacity_dev(atlasgpu_ctx* ctx, const atlasgpu_lte_line* d_lines, int64_t n,
                                     int length, int nrhox, double resolu, const float* d_cont,
                                     const double* d_xnfdop, const double* d_dopple, int nspec,
                                     const double* d_xne, const double* d_txnxn, const double* d_hckt,
                                     int maxprof, float* d_opac) {
  if (!ctx || n < 0 || length < 1 || nrhox < 1 || nrhox > kKwMax || nspec < 1 || maxprof < 1 ||
      !(resolu > 0.0) || !d_cont || !d_xnfdop || !d_dopple || !d_xne || !d_txnxn || !d_hckt ||
      !d_opac || (n > 0 && !d_lines))
    return fail(ctx, ATLASGPU_EINVAL, "synthe_line_opacity: bad argument");
  cudaSetDevice(ctx->device);
  const int ntiles = (length + kTile - 1) / kTile;
  double* acc;
  int r;
  if ((r = bufT(ctx, "lo_acc", (size_t)nrhox * length, &acc))) return r;
  CK(cudaMemsetAsync(acc, 0, (size_t)nrhox * length * sizeof(double), ctx->stream));
  const int64_t nn = n > 0 ? n : 1;
  // depth batch so that the far-line lists stay within ~4 GB
  int nj = (int)std::min<int64_t>(nrhox, std::max<int64_t>(1, (4ll << 30) / (nn * (int64_t)sizeof(FarLine))));
  FarLine* far;
  unsigned* nfar;
  int* tdiff;
  int64_t *off, *fillptr, *tot, *base;
  if ((r = bufT(ctx, "lo_far", (size_t)nj * nn, &far)) || (r = bufT(ctx, "lo_nfar", nj, &nfar)) ||
      (r = bufT(ctx, "lo_tdiff", (size_t)nj * (ntiles + 1), &tdiff)) ||
      (r = bufT(ctx, "lo_off", (size_t)nj * (ntiles + 1), &off)) ||
      (r = bufT(ctx, "lo_fill", (size_t)nj * ntiles, &fillptr)) || (r = bufT(ctx, "lo_tot", nj, &tot)) ||
      (r = bufT(ctx, "lo_base", nj, &base)))
    return r;
  std::vector<int64_t> htot(nj), hbase(nj);
  unsigned long long* work = work_counters(ctx, 4);
  // the families run once per depth batch: their times add up over the call
  if (ctx->timing)
    for (const char* f : {"synthe_core", "synthe_farfill", "synthe_farwing"}) ctx->kms[f] = 0.0;
  for (int j0 = 0; j0 < nrhox; j0 += nj) {
    const int nb = std::min(nj, nrhox - j0);
    CK(cudaMemsetAsync(nfar, 0, nb * sizeof(unsigned), ctx->stream));
    CK(cudaMemsetAsync(tdiff, 0, (size_t)nb * (ntiles + 1) * sizeof(int), ctx->stream));
    if (n > 0) {
      CoreArgs a{d_lines, n, length, nrhox, nspec, maxprof, j0, nb, resolu, d_cont, d_xnfdop,
                 d_dopple, d_xne, d_txnxn, d_hckt, acc, far, nfar, tdiff, ntiles, work};
      Timer tm(ctx, "synthe_core", true);
      const int64_t groups = n * nb;
      k_core<<<grid_for(ctx, groups, 256, 4), 256, 0, ctx->stream>>>(a);
      CKL(ctx);
    }
    k_far_scan<<<nb, 32, 0, ctx->stream>>>(tdiff, ntiles, off, fillptr, tot);
    CKL(ctx);
    CK(cudaMemcpyAsync(htot.data(), tot, nb * sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    int64_t run = 0;
    for (int k = 0; k < nb; ++k) {
      hbase[k] = run;
      run += htot[k];
    }
    int* csr;
    if ((r = bufT(ctx, "lo_csr", (size_t)std::max<int64_t>(run, 1), &csr))) return r;
    CK(cudaMemcpyAsync(base, hbase.data(), nb * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    {
      Timer tm(ctx, "synthe_farfill", true);
      dim3 g(std::max(1, std::min(ctx->nsm * 4 / std::max(1, nb) + 1, 1024)), nb);
      k_far_fill<<<g, 256, 0, ctx->stream>>>(far, nfar, nn, length, base, fillptr, ntiles, csr);
      CKL(ctx);
    }
    {
      Timer tm(ctx, "synthe_farwing", true);
      dim3 g(ntiles * kSubs, nb);
      if (ctx->precision == ATLASGPU_PREC_MIXED)
        k_farwing<true><<<g, 32, 0, ctx->stream>>>(far, nn, off, base, csr, ntiles, length, j0, acc, d_opac,
                                                            work);
      else
        k_farwing<false><<<g, 32, 0, ctx->stream>>>(far, nn, off, base, csr, ntiles, length, j0, acc, d_opac,
                                                             work);
      CKL(ctx);
    }
  }
  work_collect(ctx, work, {"synthe_voigt_evals", "synthe_farwing_updates", "synthe_farwing_expansions",
                           "synthe_farwing_direct_pairs"});
  return 0;
}

int atlasgpu_synthe_line_opacity(atlasgpu_ctx* ctx, const atlasgpu_lte_line* lines, int64_t n,
                                 int length, int nrhox, double resolu, const float* continuum,
                                 const double* xnfdop, const double* dopple, int nspec,
                                 const double* xne, const double* txnxn, const double* hckt,
                                 int maxprof, float* opacity_out) {
  if (!ctx || n < 0 || (n > 0 && !lines) || !continuum || !xnfdop || !dopple || !xne || !txnxn ||
      !hckt || !opacity_out || length < 1 || nrhox < 1 || nrhox > kKwMax || nspec < 1)
    return fail(ctx, ATLASGPU_EINVAL, "synthe_line_opacity: bad argument");
  for (int64_t i = 0; i < n; ++i)
    if (lines[i].nelion < 1 || lines[i].nelion > nspec)
      return fail(ctx, ATLASGPU_EINVAL, "line %lld: nelion %d outside 1..%d", (long long)i, lines[i].nelion, nspec);
  cudaSetDevice(ctx->device);
  atlasgpu_lte_line* d_l;
  float *d_c, *d_o;
  double *d_xd, *d_dp, *d_xne, *d_tx, *d_hc;
  int r;
  const size_t nd = (size_t)nrhox * nspec;
  if ((r = bufT(ctx, "h_lines", (size_t)std::max<int64_t>(n, 1), &d_l)) ||
      (r = bufT(ctx, "h_cont", (size_t)nrhox * length, &d_c)) ||
      (r = bufT(ctx, "h_opac", (size_t)nrhox * length, &d_o)) || (r = bufT(ctx, "h_xnfdop", nd, &d_xd)) ||
      (r = bufT(ctx, "h_dopple", nd, &d_dp)) || (r = bufT(ctx, "h_xne", nrhox, &d_xne)) ||
      (r = bufT(ctx, "h_txnxn", nrhox, &d_tx)) || (r = bufT(ctx, "h_hckt", nrhox, &d_hc)))
    return r;
  cudaStream_t s = ctx->stream;
  if (n > 0) CK(cudaMemcpyAsync(d_l, lines, n * sizeof(atlasgpu_lte_line), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_c, continuum, (size_t)nrhox * length * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xd, xnfdop, nd * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_dp, dopple, nd * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xne, xne, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_tx, txnxn, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_hc, hckt, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  if ((r = atlasgpu_synthe_line_opacity_dev(ctx, d_l, n, length, nrhox, resolu, d_c, d_xd, d_dp, nspec,
                                            d_xne, d_tx, d_hc, maxprof, d_o)))
    return r;
  CK(cudaMemcpyAsync(opacity_out, d_o, (size_t)nrhox * length * sizeof(float), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

// ---------------------------------------------------------------- spectrum
static int spectrum_launch(atlasgpu_ctx* ctx, const SpecArgs& a) {
  int nwarp = 4;
  const size_t per = sizeof(SpecWS);
  while (nwarp > 1 && sizeof(double) * kKwMax + nwarp * per > ctx->smem_optin) --nwarp;
  const size_t smem = sizeof(double) * kKwMax + nwarp * per;
  CK(cudaFuncSetAttribute(k_spectrum, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int blocks = std::min<int64_t>((a.length + nwarp - 1) / nwarp, (int64_t)ctx->nsm * 8);
  Timer tm(ctx, "josh_spectrum");
  k_spectrum<<<blocks, 32 * nwarp, smem, ctx->stream>>>(a);
  CKL(ctx);
  return 0;
}

int atlasgpu_synthe_spectrum_dev(atlasgpu_ctx* ctx, const double* d_wledge, int nedge,
                                 const double* d_contabs, const double* d_contscat, int stride,
                                 int nrhox, const double* d_rhox, const double* d_hkt, double wbegin,
                                 double ratio, int length, const float* d_opac, double* d_flux,
                                 double* d_cont) {
  if (!ctx || !ctx->ops_set) return fail(ctx, ATLASGPU_ESTATE, "synthe_spectrum: operators not set");
  if (nedge < 2 || nrhox < 4 || nrhox > kKwMax || length < 1 || stride < 3 * (nedge - 1) || !d_wledge ||
      !d_contabs || !d_contscat || !d_rhox || !d_hkt || !d_opac || !d_flux || !d_cont)
    return fail(ctx, ATLASGPU_EINVAL, "synthe_spectrum: bad argument");
  cudaSetDevice(ctx->device);
  SpecArgs a{ctx->ops, d_wledge, d_contabs, d_contscat, d_rhox, d_hkt, nedge, stride, nrhox, length,
             wbegin, ratio, d_opac, d_flux, d_cont};
  return spectrum_launch(ctx, a);
}

namespace {
// The grid indices of a merged-continuum edge at one depth
// (synthe_module.f90:3664-3689, vacuum wavelengths): NBUFF1 the first point
// redward of the line, NBUFF2 at WMERGE, NBUFF3 at WTAIL = 500 cm^-1 redder;
// WMERGE from the REAL(4) Inglis-Teller NMERGE (:3344-3347), H I with
// RYDBERG_H.  The REAL(4) edge test uses the C library expf as the
// reference's REAL(4) EXP does.  Returns 0 when the edge misses the grid.
int merged_bins(double wl, int nlast, int nelion, double xne, double wbegin, double ratio, int length, int* n1,
                int* n2, int* n3) {
  const double ratiolg = log(ratio);
  const int ixwlbeg = (int)lrint(log(wbegin) / ratiolg);
  const float inglis = (float)(1600.0 / pow(xne, (double)(2.0f / 15.0f)));
  const float nmerge = inglis - 1.5f;
  const double ryd = nelion == 1 ? 109677.583403 : 109737.31568157;  // RYDBERG_H, RYDBERG_INF
  const double em = ryd / ((double)nmerge * (double)nmerge);
  const double wshift = 1.0e7 / (1.0e7 / wl - ryd / ((double)nlast * (double)nlast));
  double wmerge = 1.0e7 / (1.0e7 / wl - em);
  if (wmerge < 0.0) wmerge = wshift + wshift;
  wmerge = std::max(wmerge, wshift);
  wmerge = std::min(wshift + wshift, wmerge);
  double wtail = 1.0e7 / (1.0e7 / wmerge - 500.0);
  if (wtail < 0.0) wtail = wmerge + wmerge;
  wtail = std::min(wmerge + wmerge, wtail);
  int ixwl = (int)(log(wl) / ratiolg);
  const float edgeblue = expf((float)ixwl * (float)ratiolg);
  if (edgeblue > (float)wl) ixwl -= 1;
  *n1 = ixwl + 1 - ixwlbeg + 1;
  *n2 = (int)(log(wmerge) / ratiolg + 0.5) - ixwlbeg + 1;
  *n3 = (int)(log(wtail) / ratiolg + 0.5) - ixwlbeg + 1;
  if (*n1 > length || *n3 < 1) return 0;
  *n1 = std::max(*n1, 1);
  return 1;
}
}  // namespace

// SYNTHE's hydrogen lines: per hydrogen record the walk's constants, and per
// (record, depth) the KAPPA0 gates, WCON/WTAIL and whose Doppler width the
// reference's SAVE'd Stehle convolution was built with (the first record of a
// run of consecutive records with the same NBLO, NBUP that reach
// hydrogen_line_profile at that depth)
static int synthe_hydrogen_launch(atlasgpu_ctx* ctx, const atlasgpu_nlte_line* recs, int64_t n, int length, int nrhox,
                                  double wbegin, double ratio, double wlend, double dopratio, const float* continuum,
                                  const double* xnfdop, const float* d_cont, const double* d_xd, const double* d_dp,
                                  int nspec, const double* xne, const double* d_xne, const double* hckt,
                                  const double* d_hc, const atlasgpu_synthe_hydrogen* hyd, double* d_acc) {
  static const double conth[15] = {109678.764, 27419.659, 12186.462, 6854.871, 4387.113, 3046.604, 2238.320, 1713.713,
                                   1354.044,   1096.776,  906.426,   761.650,  648.980,  559.579,  487.456};
  const double rydh = 109677.583403, cutoff = 1.0e-3;
  cudaStream_t s = ctx->stream;
  atlasgpu_hydrogen_tables tab;
  CK(cudaMemcpyAsync(&tab, ctx->bufs["sh_tab"].first, sizeof tab, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double ehyd[100], alphahyd[99];
  for (int k = 1; k <= 100; ++k) ehyd[k - 1] = k <= 10 ? tab.eh[k - 1] : tab.elim - rydh / ((double)k * (double)k);
  for (int k = 1; k <= 99; ++k) alphahyd[k - 1] = 1.0e7 / (ehyd[k] - ehyd[k - 1]);
  std::vector<ShRec> hr;
  std::vector<int64_t> src;
  for (int64_t i = 0; i < n; ++i) {
    const atlasgpu_nlte_line& r = recs[i];
    if (r.itype != -1 && r.itype != -2) continue;
    ShRec q;
    q.wl = r.wlvac * dopratio;
    q.alpha = alphahyd[r.nblo - 1];
    q.gf = r.gf;
    q.elo = r.elo;
    q.n = r.nblo;
    q.m = r.nbup;
    q.nbuff = r.nbuff;
    q.variant = (r.ncon == 0 || r.nbup == r.nblo + 1) ? 0 : (r.nbup == r.nblo + 2 ? 1 : 2);
    q.deut = r.itype == -2;
    hr.push_back(q);
    src.push_back(i);
  }
  const int64_t nh = (int64_t)hr.size();
  if (nh == 0) return 0;
  std::vector<ShPair> pairs((size_t)nh * nrhox);
  for (int j = 0; j < nrhox; ++j) {
    const float inglis = (float)(1600.0 / pow(xne[j], (double)(2.0f / 15.0f)));
    const float nmerge = inglis - 1.5f;
    const double emergeh = rydh / ((double)nmerge * (double)nmerge);
    const float* cont = continuum + (size_t)j * length;
    int last_n = 0, last_m = 0, last_deut = 0;
    for (int64_t k = 0; k < nh; ++k) {
      const ShRec& q = hr[k];
      const atlasgpu_nlte_line& r = recs[src[k]];
      ShPair& p = pairs[(size_t)k * nrhox + j];
      p.wcon = p.wtail = 0.0;
      p.flags = p.pad = 0;
      double kappa0 = (double)q.gf * xnfdop[(size_t)j * nspec];
      const int ick = q.nbuff < 1 ? 1 : (q.nbuff > length ? length : q.nbuff);
      const double kapmin = (double)cont[(q.m == 2 ? length : ick) - 1] * cutoff;
      if (kappa0 < kapmin) continue;
      kappa0 = kappa0 * exp(-(double)q.elo * hckt[j]);
      if (kappa0 < kapmin) continue;
      p.flags = 1;
      if (q.variant == 2) {
        const double wshift = 1.0e7 / (conth[r.ncon - 1] - rydh / (81.0 * 81.0));
        double wmerge = 1.0e7 / (conth[r.ncon - 1] - emergeh);
        if (wmerge < 0.0) wmerge = wshift + wshift;
        double wcon = wshift > wmerge ? wshift : wmerge;
        double wtail = 1.0e7 / (1.0e7 / wcon - 500.0);
        if (wshift + wshift < wcon) wcon = wshift + wshift;
        if (wtail < 0.0) wtail = wcon + wcon;
        if (wcon + wcon < wtail) wtail = wcon + wcon;
        p.wcon = wcon * dopratio;
        p.wtail = wtail;
      }
      // does the walk reach hydrogen_line_profile at all?
      const int minred = q.nbuff > 1 ? q.nbuff : 1;
      const int ib0 = q.nbuff < length + 1 ? q.nbuff : length + 1;
      bool calls = false, blue = true;
      if (q.variant == 0) {
        if (q.wl <= wlend) {
          calls = minred <= length;
          if (minred == 1 || q.wl < wbegin) blue = false;
        }
      } else if (q.variant == 1) {
        if (q.wl <= wlend) {
          if (minred <= length) {
            if (!(wbegin * powi(ratio, minred - 1) > q.alpha)) calls = true;
          } else if (minred == 1 || q.wl < wbegin || q.nbuff < 1) {
            blue = false;
          }
        } else if (q.nbuff < 1) {
          blue = false;
        }
      } else {
        blue = false;
        if (!(q.wl <= wlend && p.wcon > wlend)) {
          bool skip = false;
          if (q.wl <= wlend) {
            if (wbegin <= q.alpha) {
              if (wbegin * powi(ratio, minred - 1) >= p.wcon) calls = true;
              else if (minred == 1) skip = true;
            }
            if (!calls && !skip && q.wl < wbegin) skip = true;
          }
          if (!calls && !skip && ib0 - 1 >= 1 && !(wbegin * powi(ratio, ib0 - 1) / ratio < p.wcon)) calls = true;
        }
      }
      if (!calls && blue && ib0 - 1 >= 1) calls = true;
      if (!calls) continue;
      if (q.n == last_n && q.m == last_m) {
        if (last_deut) p.flags |= 2;
      } else {
        last_n = q.n;
        last_m = q.m;
        last_deut = q.deut;
        if (q.deut) p.flags |= 2;
      }
    }
  }
  ShRec* d_hr;
  ShPair* d_pair;
  double* d_hv;
  int r;
  if ((r = bufT(ctx, "sh_rec", (size_t)nh, &d_hr)) || (r = bufT(ctx, "sh_pair", pairs.size(), &d_pair)) ||
      (r = bufT(ctx, "sh_hv", (size_t)5 * nrhox, &d_hv)))
    return r;
  CK(cudaMemcpyAsync(d_hr, hr.data(), (size_t)nh * sizeof(ShRec), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_pair, pairs.data(), pairs.size() * sizeof(ShPair), cudaMemcpyHostToDevice, s));
  const double* hv[5] = {hyd->t, hyd->xnfph1, hyd->xnfph2, hyd->xnfhe1, hyd->xnfh2};
  for (int q = 0; q < 5; ++q)
    CK(cudaMemcpyAsync(d_hv + (size_t)q * nrhox, hv[q], nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  ShArgs a{d_hr, d_pair, nh, nrhox, length, nspec, wbegin, ratio, wlend, d_cont, d_xd, d_dp, d_xne, d_hc,
           d_hv, d_hv + nrhox, d_hv + 2 * nrhox, d_hv + 3 * nrhox, d_hv + 4 * nrhox,
           (const atlasgpu_hydrogen_tables*)ctx->bufs["sh_tab"].first,
           (const StehleDev*)ctx->bufs["sh_stehle"].first, d_acc};
  const int64_t nwarps = nh * nrhox;
  const int blocks = grid_for(ctx, nwarps * 32, 32 * kShWarps, 32);
  k_synthe_hydrogen<<<blocks, 32 * kShWarps, 0, s>>>(a);
  CKL(ctx);
  CK(cudaStreamSynchronize(s));  // the host vectors go out of scope
  return 0;
}

}  // extern "C"

namespace atlasgpu {

// The four Stehle series into device buffers named <prefix>_mdi<q>,
// <prefix>_ka<q>, <prefix>_pr<q> and the StehleDev array <prefix> (NULL or a
// series with n_dens 0: not loaded); *out the device array.  Validates first.
int stehle_upload(atlasgpu_ctx* ctx, const atlasgpu_stehle_series* stehle, const char* prefix, const char* who,
                  StehleDev** out) {
  StehleDev dev[4] = {};
  if (stehle) {
    for (int q = 0; q < 4; ++q) {
      const atlasgpu_stehle_series& S = stehle[q];
      if (S.n_dens == 0) continue;
      const int ntr = S.n_upper_max - S.n_upper_min + 1;
      if (S.n_lower != q + 1 || S.n_upper_min <= S.n_lower || ntr < 1 || S.n_upper_max > 100 || S.n_dens < 2 ||
          S.n_dens > 20 || !S.max_dens_idx || !S.k_alpha || !S.profiles)
        return fail(ctx, ATLASGPU_EINVAL, "%s: Stehle series %d malformed", who, q + 1);
      for (int t = 0; t < ntr; ++t)
        if (S.max_dens_idx[t] < 1 || S.max_dens_idx[t] > S.n_dens)
          return fail(ctx, ATLASGPU_EINVAL, "%s: Stehle series %d density index", who, q + 1);
    }
  }
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  StehleDev* d_st;
  int r;
  if ((r = bufT(ctx, prefix, 4, &d_st))) return r;
  for (int q = 0; stehle && q < 4; ++q) {
    const atlasgpu_stehle_series& S = stehle[q];
    StehleDev& D = dev[q];
    if (S.n_dens == 0) continue;
    const int ntr = S.n_upper_max - S.n_upper_min + 1;
    const size_t np = (size_t)ntr * S.n_dens * 600;
    char nm[3][48];
    snprintf(nm[0], sizeof nm[0], "%s_mdi%d", prefix, q);
    snprintf(nm[1], sizeof nm[1], "%s_ka%d", prefix, q);
    snprintf(nm[2], sizeof nm[2], "%s_pr%d", prefix, q);
    int32_t* d_mdi;
    double *d_ka, *d_pr;
    if ((r = bufT(ctx, nm[0], (size_t)ntr, &d_mdi)) || (r = bufT(ctx, nm[1], (size_t)ntr, &d_ka)) ||
        (r = bufT(ctx, nm[2], np, &d_pr)))
      return r;
    CK(cudaMemcpyAsync(d_mdi, S.max_dens_idx, ntr * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_ka, S.k_alpha, ntr * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_pr, S.profiles, np * sizeof(double), cudaMemcpyHostToDevice, s));
    D.n_lower = S.n_lower;
    D.n_upper_min = S.n_upper_min;
    D.n_upper_max = S.n_upper_max;
    D.n_dens = S.n_dens;
    memcpy(D.density_grid, S.density_grid, sizeof D.density_grid);
    memcpy(D.temp_grid, S.temp_grid, sizeof D.temp_grid);
    memcpy(D.log_dalpha_grid, S.log_dalpha_grid, sizeof D.log_dalpha_grid);
    D.max_dens_idx = d_mdi;
    D.k_alpha = d_ka;
    D.profiles = d_pr;
  }
  CK(cudaMemcpyAsync(d_st, dev, sizeof dev, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  *out = d_st;
  return 0;
}

}  // namespace atlasgpu

extern "C" {

int atlasgpu_synthe_set_hydrogen_tables(atlasgpu_ctx* ctx, const atlasgpu_hydrogen_tables* tables,
                                        const atlasgpu_stehle_series* stehle) {
  if (!ctx || !tables) return fail(ctx, ATLASGPU_EINVAL, "synthe_set_hydrogen_tables: null argument");
  for (int q = 0; q < 4; ++q)
    if (tables->lnghal[q] < 1 || tables->lnghal[q] > 14 || tables->istal[q] < 1 ||
        tables->istal[q] + tables->lnghal[q] - 1 > 34 || tables->lncomp[q] < 1 || tables->lncomp[q] > 5)
      return fail(ctx, ATLASGPU_EINVAL, "synthe_set_hydrogen_tables: fine-structure index out of range");
  StehleDev* d_st;
  int r;
  if ((r = stehle_upload(ctx, stehle, "sh_stehle", "synthe_set_hydrogen_tables", &d_st))) return r;
  atlasgpu_hydrogen_tables* d_tab;
  if ((r = bufT(ctx, "sh_tab", 1, &d_tab))) return r;
  CK(cudaMemcpyAsync(d_tab, tables, sizeof *tables, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int atlasgpu_synthe_nlte_opacity(atlasgpu_ctx* ctx, const atlasgpu_nlte_line* recs, int64_t n, int length,
                                 int nrhox, double wbegin, double ratio, double wlend, double velshift_kms,
                                 const float* continuum, const double* xnfdop, const double* dopple,
                                 const double* xnfpel, int nspec, const double* xne, const double* txnxn,
                                 const double* hckt, const double* contx, const atlasgpu_synthe_hydrogen* hyd,
                                 float* opacity_inout) {
  if (!ctx || n < 0 || (n > 0 && !recs) || length < 1 || nrhox < 1 || nrhox > kKwMax || !(wbegin > 0.0) ||
      !(ratio > 1.0) || !continuum || !xnfdop || !dopple || nspec < 1 || !xne || !txnxn || !hckt || !contx ||
      !opacity_inout)
    return fail(ctx, ATLASGPU_EINVAL, "synthe_nlte_opacity: bad argument");
  if (hyd) {
    if (!hyd->t || !hyd->xnfph1 || !hyd->xnfph2 || !hyd->xnfhe1 || !hyd->xnfh2)
      return fail(ctx, ATLASGPU_EINVAL, "synthe_nlte_opacity: hydrogen lines need T, XNFPH, XNFHE, XNFH2");
    if (ctx->bufs.find("sh_tab") == ctx->bufs.end())
      return fail(ctx, ATLASGPU_ESTATE, "synthe_nlte_opacity: hydrogen tables not set");
    for (int64_t i = 0; i < n; ++i) {
      const atlasgpu_nlte_line& r = recs[i];
      if ((r.itype == -1 || r.itype == -2) &&
          (r.nblo < 1 || r.nblo > 99 || r.nbup <= r.nblo || r.nbup > 100 || r.ncon < 0 || r.ncon > 15))
        return fail(ctx, ATLASGPU_EINVAL, "synthe_nlte_opacity: hydrogen record %lld has NBLO %d NBUP %d NCON %d",
                    (long long)i, r.nblo, r.nbup, r.ncon);
    }
  }
  for (int64_t i = 0; i < n; ++i) {
    const int t = recs[i].itype;
    const bool normal = t == 0 || t == 3 || t <= -3;
    if (normal && recs[i].ncon > 0 && (recs[i].ncon > 26 || recs[i].nelionx < 1 || recs[i].nelionx > 17))
      return fail(ctx, ATLASGPU_EINVAL, "synthe_nlte_opacity: NCON %d / NELIONX %d outside CONTX at record %lld",
                  recs[i].ncon, recs[i].nelionx, (long long)i);
  }
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t nm = (size_t)nrhox * length, nd = (size_t)nrhox * nspec;
  atlasgpu_nlte_line* d_rec;
  float *d_cont, *d_op;
  double *d_xd, *d_dp, *d_xne, *d_tx, *d_hc, *d_em, *d_cx, *d_acc;
  int r;
  if ((r = bufT(ctx, "sn_rec", (size_t)std::max<int64_t>(n, 1), &d_rec)) || (r = bufT(ctx, "sn_cont", nm, &d_cont)) ||
      (r = bufT(ctx, "sn_op", nm, &d_op)) || (r = bufT(ctx, "sn_xd", nd, &d_xd)) || (r = bufT(ctx, "sn_dp", nd, &d_dp)) ||
      (r = bufT(ctx, "sn_xne", nrhox, &d_xne)) || (r = bufT(ctx, "sn_tx", nrhox, &d_tx)) ||
      (r = bufT(ctx, "sn_hc", nrhox, &d_hc)) || (r = bufT(ctx, "sn_em", nrhox, &d_em)) ||
      (r = bufT(ctx, "sn_cx", 26 * 17, &d_cx)) || (r = bufT(ctx, "sn_acc", nm, &d_acc)))
    return r;
  // EMERGE(J) = RYDBERG_INF / NMERGE**2 with the reference's REAL(4) INGLIS and NMERGE = INGLIS - 1.5
  std::vector<double> em(nrhox);
  for (int j = 0; j < nrhox; ++j) {
    const float inglis = (float)(1600.0 / pow(xne[j], (double)(2.0f / 15.0f)));
    const float nmerge = inglis - 1.5f;
    em[j] = 109737.31568157 / ((double)nmerge * (double)nmerge);
  }
  if (n > 0) CK(cudaMemcpyAsync(d_rec, recs, n * sizeof(atlasgpu_nlte_line), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_cont, continuum, nm * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_op, opacity_inout, nm * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xd, xnfdop, nd * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_dp, dopple, nd * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_xne, xne, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_tx, txnxn, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_hc, hckt, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_em, em.data(), nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_cx, contx, 26 * 17 * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(d_acc, 0, nm * sizeof(double), s));
  if (n > 0) {
    NlteArgs a{d_rec, n, length, nrhox, nspec, wbegin, ratio, wlend, 1.0 + velshift_kms / 299792.458, d_cont, d_xd,
               d_dp, d_xne, d_tx, d_hc, d_em, d_cx, d_acc};
    if (xnfpel) {
      double* d_xp;
      if ((r = bufT(ctx, "sn_xp", nd, &d_xp))) return r;
      CK(cudaMemcpyAsync(d_xp, xnfpel, nd * sizeof(double), cudaMemcpyHostToDevice, s));
      a.xnfpel = d_xp;
      // merged-continuum edges: their grid indices per depth, from the C library
      std::vector<int> mord((size_t)n, -1);
      std::vector<int4> mb;
      const double dopratio = a.dopratio;
      for (int64_t i = 0; i < n; ++i) {
        const atlasgpu_nlte_line& rec = recs[i];
        if (rec.itype < 4 || rec.nelion < 1 || rec.nelion > nspec) continue;
        mord[i] = (int)(mb.size() / nrhox);
        for (int j = 0; j < nrhox; ++j) {
          int4 b;
          b.w = merged_bins(rec.wlvac * dopratio, rec.itype, rec.nelion, xne[j], wbegin, ratio, length, &b.x, &b.y,
                            &b.z);
          mb.push_back(b);
        }
      }
      if (!mb.empty()) {
        int* d_mo;
        int4* d_mb;
        if ((r = bufT(ctx, "sn_mord", (size_t)n, &d_mo)) || (r = bufT(ctx, "sn_mbins", mb.size(), &d_mb))) return r;
        CK(cudaMemcpyAsync(d_mo, mord.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_mb, mb.data(), mb.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));  // the host vectors go out of scope
        a.mord = d_mo;
        a.mbins = d_mb;
      }
    }
    Timer tm(ctx, "synthe_nlte");
    k_synthe_nlte<<<grid_for(ctx, n * nrhox * 32, 256, 16), 256, 0, s>>>(a);
    CKL(ctx);
    if (hyd && (r = synthe_hydrogen_launch(ctx, recs, n, length, nrhox, wbegin, ratio, wlend, a.dopratio, continuum,
                                           xnfdop, d_cont, d_xd, d_dp, nspec, xne, d_xne, hckt, d_hc, hyd, d_acc)))
      return r;
    k_add_f64_to_f32<<<grid_for(ctx, (int64_t)nm, 256, 8), 256, 0, s>>>(d_acc, d_op, (int64_t)nm);
    CKL(ctx);
  }
  CK(cudaMemcpyAsync(opacity_inout, d_op, nm * sizeof(float), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int atlasgpu_synthe_spectrum(atlasgpu_ctx* ctx, const double* wledge, int nedge, const double* contabs,
                             const double* contscat, int stride, int nrhox, const double* rhox,
                             const double* hkt, double wbegin, double ratio, int length,
                             const float* opacity, double* flux, double* cont) {
  if (!ctx || !wledge || !contabs || !contscat || !rhox || !hkt || !opacity || !flux || !cont ||
      nedge < 2 || nrhox < 4 || nrhox > kKwMax || length < 1 || stride < 3 * (nedge - 1))
    return fail(ctx, ATLASGPU_EINVAL, "synthe_spectrum: bad argument");
  for (int i = 1; i < nedge; ++i)
    if (!(wledge[i] > wledge[i - 1])) return fail(ctx, ATLASGPU_EINVAL, "wledge not increasing");
  if (!finite_all(contabs, (size_t)nrhox * stride) || !finite_all(contscat, (size_t)nrhox * stride) ||
      !finite_all(rhox, nrhox) || !finite_all(hkt, nrhox))
    return fail(ctx, ATLASGPU_ENONFINITE, "synthe_spectrum: non-finite input");
  cudaSetDevice(ctx->device);
  double *d_we, *d_ca, *d_cs, *d_rx, *d_hk, *d_fl, *d_ct;
  float* d_op;
  int r;
  const size_t nt = (size_t)nrhox * stride;
  if ((r = bufT(ctx, "s_we", nedge, &d_we)) || (r = bufT(ctx, "s_ca", nt, &d_ca)) ||
      (r = bufT(ctx, "s_cs", nt, &d_cs)) || (r = bufT(ctx, "s_rx", nrhox, &d_rx)) ||
      (r = bufT(ctx, "s_hk", nrhox, &d_hk)) || (r = bufT(ctx, "s_fl", length, &d_fl)) ||
      (r = bufT(ctx, "s_ct", length, &d_ct)) || (r = bufT(ctx, "s_op", (size_t)nrhox * length, &d_op)))
    return r;
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(d_we, wledge, nedge * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_ca, contabs, nt * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_cs, contscat, nt * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_rx, rhox, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_hk, hkt, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_op, opacity, (size_t)nrhox * length * sizeof(float), cudaMemcpyHostToDevice, s));
  if ((r = atlasgpu_synthe_spectrum_dev(ctx, d_we, nedge, d_ca, d_cs, stride, nrhox, d_rx, d_hk, wbegin,
                                        ratio, length, d_op, d_fl, d_ct)))
    return r;
  CK(cudaMemcpyAsync(flux, d_fl, length * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(cont, d_ct, length * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

}  // extern "C"
