// api_kapp.cu -- C-ABI entry points of KAPP's hydrogen, helium and H2
// continuum sources (atlas12_modules.f90:11202-11324 with HOP, H2PLOP, HMINOP,
// HRAYOP, ELECOP, HE1OP, HE2OP, HEMIOP, HERAOP, H2MINOP, H2COLLOP, H2RAOP)
// and of HLINOP's hydrogen line pseudo-continuum; kernels in kapp.cuh.
#include <cmath>
#include <vector>

#include "api_common.cuh"
#include "kapp.cuh"

using namespace atlasgpu;

namespace {

// H_SERIES_LIMITS (atlas12_modules.f90:392-395): HOP's cascade exits at the
// same thresholds as the reference's
constexpr double kSeriesLimits[15] = {109678.764, 27419.659, 12186.462, 6854.871, 4387.113,
                                      3046.604,   2238.320,  1713.713,  1354.044, 1096.776,
                                      906.426,    761.650,   648.980,   559.579,  487.456};

bool finite_f(const float* p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

}  // namespace

extern "C" {

int atlasgpu_atlas_set_kapp_tables(atlasgpu_ctx* ctx, const atlasgpu_kapp_tables* t) {
  if (!ctx || !t) return fail(ctx, ATLASGPU_EINVAL, "set_kapp_tables: null argument");
  if (!finite_f(&t->freqn[0][0], 15 * 29) || !finite_f(&t->xn[0][0], 15 * 29) || !finite_f(&t->xl[0][0][0], 36 * 29) ||
      !finite_f(t->ekarzas, 29) || !finite_all(&t->gff[0][0], 146 * 81) || !finite_all(t->q_holtsmark, 150) ||
      !finite_all(t->hop_elev, 15) || !finite_all(t->hmin_wbf, 116) || !finite_all(t->hmin_bf, 116) ||
      !finite_all(t->hmin_thetaff, 11) || !finite_all(t->hmin_wavek, 22) || !finite_all(&t->hmin_ff[0][0], 242) ||
      !finite_all(t->h2p_fr, 5) || !finite_all(t->h2p_es, 6) || !finite_all(t->ray_m, 74) ||
      !finite_all(t->ray_ab, 27) || !finite_all(t->ray_bc, 24) || !finite_all(t->ray_cd, 22) ||
      !finite_all(t->ray_ly, 64) || !finite_all(t->ray_fly, 64) || !finite_all(t->he1_chi, 10) ||
      !finite_all(t->he1_freq, 10) || !finite_all(t->he1_g, 10) || !finite_all(t->he_x505, 92) ||
      !finite_all(t->he_x50, 16) || !finite_all(t->he_x20, 11) || !finite_all(t->he_x10, 21) ||
      !finite_all(t->he2s1s_f, 16) || !finite_all(t->he2s1s_x, 16) || !finite_all(t->he2s3s_f, 16) ||
      !finite_all(t->he2s3s_x, 16) || !finite_all(t->he2p1p_f, 16) || !finite_all(t->he2p1p_x, 16) ||
      !finite_all(t->he2p3p_f, 16) || !finite_all(t->he2p3p_x, 16) || !finite_all(t->hem_w, 17) ||
      !finite_all(t->hem_t, 12) || !finite_all(&t->hem_k[0][0], 12 * 17) || !finite_all(t->gf_lyman, 29) ||
      !finite_all(t->gf_balmer, 28) || !finite_all(t->gf_paschen, 27) || !finite_all(t->gf_brackett, 3) ||
      !finite_all(&t->stark_knm[0][0], 20) || !finite_all(&t->stark_f[0][0], 40))
    return fail(ctx, ATLASGPU_ENONFINITE, "set_kapp_tables: non-finite table entry");
  for (int i = 0; i < 12 * 17; ++i)
    if (!((&t->hem_k[0][0])[i] > 0.0)) return fail(ctx, ATLASGPU_EINVAL, "set_kapp_tables: KHEM entry not positive");
  for (int i = 0; i < 17; ++i)
    if (!(t->hem_w[i] > 0.0) || (i > 0 && !(t->hem_w[i] > t->hem_w[i - 1])))
      return fail(ctx, ATLASGPU_EINVAL, "set_kapp_tables: WHEM not positive and increasing");
  for (int i = 0; i < 12; ++i)
    if (!(t->hem_t[i] > 0.0) || (i > 0 && !(t->hem_t[i] > t->hem_t[i - 1])))
      return fail(ctx, ATLASGPU_EINVAL, "set_kapp_tables: THEM not positive and increasing");
  for (int i = 0; i < 146 * 81; ++i)
    if (!((&t->gff[0][0])[i] > 0.0)) return fail(ctx, ATLASGPU_EINVAL, "set_kapp_tables: g_ff entry not positive");
  for (int i = 0; i < 242; ++i)
    if (!((&t->hmin_ff[0][0])[i] > 0.0)) return fail(ctx, ATLASGPU_EINVAL, "set_kapp_tables: FF entry not positive");
  for (int i = 0; i < 22; ++i)
    if (!(t->hmin_wavek[i] > 0.0)) return fail(ctx, ATLASGPU_EINVAL, "set_kapp_tables: WAVEK entry not positive");
  std::vector<KappDev> h(1);
  KappDev& k = h[0];
  std::copy(&t->freqn[0][0], &t->freqn[0][0] + 15 * 29, k.freqn);
  std::copy(&t->xn[0][0], &t->xn[0][0] + 15 * 29, k.xn);
  std::copy(&t->xl[0][0][0], &t->xl[0][0][0] + 36 * 29, k.xl);
  std::copy(t->ekarzas, t->ekarzas + 29, k.ekarzas);
  // COULFF's reader (:12162-12165): GFF_LOGTAB = log10 of the tabulated g_ff
  for (int i = 0; i < 146 * 81; ++i) k.gff_log[i] = std::log10((&t->gff[0][0])[i]);
  std::copy(t->q_holtsmark, t->q_holtsmark + 150, k.q);
  std::copy(t->hop_elev, t->hop_elev + 15, k.hop_elev);
  std::copy(t->hmin_wbf, t->hmin_wbf + 116, k.wbf);
  std::copy(t->hmin_bf, t->hmin_bf + 116, k.bf);
  std::copy(t->hmin_thetaff, t->hmin_thetaff + 11, k.thetaff);
  // HMINOP's first call (:12488-12497): WFFLOG = log(91.134 / WAVEK),
  // FFLOG(IWAVE, ITHETA) = log(FF(ITHETA, IWAVE) * 1e-26)
  for (int iw = 0; iw < 22; ++iw) {
    k.wfflog[iw] = std::log(91.134 / t->hmin_wavek[iw]);
    for (int it = 0; it < 11; ++it) k.fflog[it * 22 + iw] = std::log(t->hmin_ff[iw][it] * 1.0e-26);
  }
  std::copy(t->h2p_fr, t->h2p_fr + 5, k.h2p_fr);
  std::copy(t->h2p_es, t->h2p_es + 6, k.h2p_es);
  std::copy(t->ray_m, t->ray_m + 74, k.ray_m);
  std::copy(t->ray_ab, t->ray_ab + 27, k.ray_ab);
  std::copy(t->ray_bc, t->ray_bc + 24, k.ray_bc);
  std::copy(t->ray_cd, t->ray_cd + 22, k.ray_cd);
  std::copy(t->ray_ly, t->ray_ly + 64, k.ray_ly);
  std::copy(t->ray_fly, t->ray_fly + 64, k.ray_fly);
  std::copy(kSeriesLimits, kSeriesLimits + 15, k.series_limits);
  std::copy(t->gf_lyman, t->gf_lyman + 29, k.gf_lyman);
  std::copy(t->gf_balmer, t->gf_balmer + 28, k.gf_balmer);
  std::copy(t->gf_paschen, t->gf_paschen + 27, k.gf_paschen);
  std::copy(t->gf_brackett, t->gf_brackett + 3, k.gf_brackett);
  std::copy(&t->stark_knm[0][0], &t->stark_knm[0][0] + 20, k.stark_knm);
  std::copy(&t->stark_f[0][0], &t->stark_f[0][0] + 40, k.stark_f);
  std::copy(t->he1_chi, t->he1_chi + 10, k.he1_chi);
  std::copy(t->he1_freq, t->he1_freq + 10, k.he1_freq);
  std::copy(t->he1_g, t->he1_g + 10, k.he1_g);
  std::copy(t->he_x505, t->he_x505 + 92, k.he_x505);
  std::copy(t->he_x50, t->he_x50 + 16, k.he_x50);
  std::copy(t->he_x20, t->he_x20 + 11, k.he_x20);
  std::copy(t->he_x10, t->he_x10 + 21, k.he_x10);
  const double* knots[8] = {t->he2s1s_f, t->he2s1s_x, t->he2s3s_f, t->he2s3s_x,
                            t->he2p1p_f, t->he2p1p_x, t->he2p3p_f, t->he2p3p_x};
  double* kd[8] = {k.he2s1s_f, k.he2s1s_x, k.he2s3s_f, k.he2s3s_x, k.he2p1p_f, k.he2p1p_x, k.he2p3p_f, k.he2p3p_x};
  for (int q = 0; q < 8; ++q) std::copy(knots[q], knots[q] + 16, kd[q]);
  // HEMIOP's first call (:13788-13798): LOGW, LOGT, LOGK = log of the table
  std::copy(t->hem_w, t->hem_w + 17, k.hem_w);
  std::copy(t->hem_t, t->hem_t + 12, k.hem_t);
  for (int i = 0; i < 17; ++i) k.hem_logw[i] = std::log(t->hem_w[i]);
  for (int i = 0; i < 12; ++i) k.hem_logt[i] = std::log(t->hem_t[i]);
  for (int i = 0; i < 12 * 17; ++i) k.hem_logk[i] = std::log((&t->hem_k[0][0])[i]);
  cudaSetDevice(ctx->device);
  KappDev* d;
  int r;
  if ((r = bufT(ctx, "kapp_tab", 1, &d))) return r;
  CK(cudaMemcpyAsync(d, &k, sizeof k, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->kapp_set = true;
  return 0;
}

int atlasgpu_atlas_set_kapp_h2_tables(atlasgpu_ctx* ctx, const atlasgpu_kapp_h2_tables* t) {
  if (!ctx || !t) return fail(ctx, ATLASGPU_EINVAL, "set_kapp_h2_tables: null argument");
  if (t->pf_n < 3 || t->pf_n > 100000 || !t->pf || !(t->pf_tstep > 0.0) || !std::isfinite(t->pf_tstart) ||
      t->cia_nnu < 2 || t->cia_ntmax < 2 || !t->cia_temp || !t->cia_tab || !(t->cia_dnu > 0.0) ||
      !std::isfinite(t->cia_nu0) || (size_t)t->cia_nnu * t->cia_ntmax * 4 > ((size_t)1 << 27))
    return fail(ctx, ATLASGPU_EINVAL, "set_kapp_h2_tables: bad sizes (pf_n %d, cia %d x %d)", t->pf_n, t->cia_ntmax,
                t->cia_nnu);
  for (int p = 0; p < 4; ++p)
    if (t->cia_nt[p] < 2 || t->cia_nt[p] > t->cia_ntmax)
      return fail(ctx, ATLASGPU_EINVAL, "set_kapp_h2_tables: pair %d has %d temperatures", p + 1, t->cia_nt[p]);
  const size_t ntab = (size_t)4 * t->cia_ntmax * t->cia_nnu;
  if (!finite_all(t->h2m_w, 10) || !finite_all(t->h2m_t, 7) || !finite_all(&t->h2m_k[0][0], 70) ||
      !finite_all(t->pf, t->pf_n) || !finite_all(t->cia_temp, (size_t)4 * t->cia_ntmax) ||
      !finite_all(t->cia_tab, ntab))
    return fail(ctx, ATLASGPU_ENONFINITE, "set_kapp_h2_tables: non-finite table entry");
  for (int i = 0; i < 70; ++i)
    if (!((&t->h2m_k[0][0])[i] > 0.0)) return fail(ctx, ATLASGPU_EINVAL, "set_kapp_h2_tables: KH2M entry not positive");
  for (int i = 0; i < 10; ++i)
    if (!(t->h2m_w[i] > 0.0) || (i > 0 && !(t->h2m_w[i] > t->h2m_w[i - 1])))
      return fail(ctx, ATLASGPU_EINVAL, "set_kapp_h2_tables: WH2M not positive and increasing");
  for (int i = 0; i < 7; ++i)
    if (!(t->h2m_t[i] > 0.0) || (i > 0 && !(t->h2m_t[i] > t->h2m_t[i - 1])))
      return fail(ctx, ATLASGPU_EINVAL, "set_kapp_h2_tables: TH2M not positive and increasing");
  for (int p = 0; p < 4; ++p)
    for (int i = 1; i < t->cia_nt[p]; ++i)
      if (!(t->cia_temp[(size_t)p * t->cia_ntmax + i] > t->cia_temp[(size_t)p * t->cia_ntmax + i - 1]))
        return fail(ctx, ATLASGPU_EINVAL, "set_kapp_h2_tables: CIA temperatures of pair %d not increasing", p + 1);
  std::vector<KappH2Dev> hv(1);
  KappH2Dev& h = hv[0];
  std::copy(t->h2m_w, t->h2m_w + 10, h.h2m_w);
  std::copy(t->h2m_t, t->h2m_t + 7, h.h2m_t);
  // H2MINOP's first call (:12650-12660): LOGW, LOGT, LOGK
  for (int i = 0; i < 10; ++i) h.h2m_logw[i] = std::log(t->h2m_w[i]);
  for (int i = 0; i < 7; ++i) h.h2m_logt[i] = std::log(t->h2m_t[i]);
  for (int i = 0; i < 70; ++i) h.h2m_logk[i] = std::log((&t->h2m_k[0][0])[i]);
  h.pf_n = t->pf_n;
  h.pf_tstart = t->pf_tstart;
  h.pf_tstep = t->pf_tstep;
  h.cia_nnu = t->cia_nnu;
  h.cia_ntmax = t->cia_ntmax;
  for (int p = 0; p < 4; ++p) {
    h.cia_nt[p] = t->cia_nt[p];
    h.use_pair[p] = t->use_pair[p] ? 1 : 0;
  }
  h.cia_nu0 = t->cia_nu0;
  h.cia_dnu = t->cia_dnu;
  h.cia_numax = t->cia_nu0 + t->cia_dnu * (double)(t->cia_nnu - 1);  // CIANUMAX (:16408)
  // EQUILH2's PARAMETERs (:22449-22455)
  const double mh = 1.008 * kAmu;
  h.equil_d0 = 36118.11 * (kHplanck * kClight / kKbol);
  h.equil_pref = std::pow(2.0, 1.5) / 4.0 / std::pow(2.0 * kPi * mh * kKbol / (kHplanck * kHplanck), 1.5);
  // PARTFNH2's natural cubic spline (:22370-22384)
  const int n = t->pf_n;
  std::vector<double> pf2(n, 0.0), cwk(n, 0.0);
  const double* pf = t->pf;
  for (int k = 2; k <= n - 1; ++k) {
    pf2[k - 1] = (6.0 * (pf[k] - 2.0 * pf[k - 1] + pf[k - 2]) / (t->pf_tstep * t->pf_tstep) - pf2[k - 2]) /
                 (4.0 - cwk[k - 2]);
    cwk[k - 1] = 1.0 / (4.0 - cwk[k - 2]);
  }
  for (int k = n - 1; k >= 2; --k) pf2[k - 1] = pf2[k - 1] - cwk[k - 1] * pf2[k];
  cudaSetDevice(ctx->device);
  const size_t nd = 2 * (size_t)n + (size_t)4 * t->cia_ntmax + ntab;
  double* d;
  KappH2Dev* dh;
  int r;
  if ((r = bufT(ctx, "kapp_h2_data", nd, &d)) || (r = bufT(ctx, "kapp_h2_tab", 1, &dh))) return r;
  h.pf = d;
  h.pf2 = d + n;
  h.cia_temp = d + 2 * (size_t)n;
  h.cia_tab = d + 2 * (size_t)n + (size_t)4 * t->cia_ntmax;
  CK(cudaMemcpyAsync((void*)h.pf, pf, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync((void*)h.pf2, pf2.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync((void*)h.cia_temp, t->cia_temp, (size_t)4 * t->cia_ntmax * sizeof(double),
                     cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync((void*)h.cia_tab, t->cia_tab, ntab * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dh, &h, sizeof h, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->kapp_h2_set = true;
  return 0;
}

}  // extern "C"

namespace {

// both entry points: validate, stage the depth vectors, launch the two
// kernels, copy the totals (and the per-source parts) back
int kapp_run(atlasgpu_ctx* ctx, const char* name, int numnu, const double* waveset, int nrhox, int kw,
             const atlasgpu_kapp_pops& pp, bool helium, double* acont, double* sigmac, double* scont, double* parts) {
  if (!ctx) return ATLASGPU_EINVAL;
  if (!ctx->kapp_set) return fail(ctx, ATLASGPU_ESTATE, "%s: tables not set", name);
  const bool h2 = helium && pp.xnf_he1;
  if (h2 && !ctx->kapp_h2_set) return fail(ctx, ATLASGPU_ESTATE, "%s: H2 tables not set", name);
  if (numnu < 1 || nrhox < 1 || kw < nrhox || !waveset || !pp.t || !pp.xne || !pp.rho || !pp.xnfp_h1 ||
      !pp.xnfp_h2 || !acont || !sigmac || !scont ||
      (helium && (!pp.xnfp_he1 || !pp.xnfp_he2 || !pp.xnfp_he3 || !pp.xnf_he2)))
    return fail(ctx, ATLASGPU_EINVAL, "%s: bad argument (numnu %d, nrhox %d, kw %d)", name, numnu, nrhox, kw);
  for (int i = 0; i < numnu; ++i)
    if (!(waveset[i] > 0.0) || !std::isfinite(waveset[i]))
      return fail(ctx, ATLASGPU_EINVAL, "%s: WAVESET(%d) = %g", name, i + 1, waveset[i]);
  if (!finite_all(pp.t, nrhox) || !finite_all(pp.xne, nrhox) || !finite_all(pp.rho, nrhox) ||
      !finite_all(pp.xnfp_h1, nrhox) || !finite_all(pp.xnfp_h2, nrhox) || (pp.bmin && !finite_all(pp.bmin, nrhox)) ||
      (helium && (!finite_all(pp.xnfp_he1, nrhox) || !finite_all(pp.xnfp_he2, nrhox) ||
                  !finite_all(pp.xnfp_he3, nrhox) || !finite_all(pp.xnf_he2, nrhox))) ||
      (h2 && !finite_all(pp.xnf_he1, nrhox)))
    return fail(ctx, ATLASGPU_ENONFINITE, "%s: non-finite depth vector", name);
  for (int j = 0; j < nrhox; ++j)
    if (!(pp.t[j] > 0.0) || !(pp.rho[j] > 0.0))
      return fail(ctx, ATLASGPU_EINVAL, "%s: T or RHO not positive at depth %d", name, j + 1);
  if (pp.bhyd)
    for (int n = 0; n < 6; ++n)
      if (!finite_all(pp.bhyd + (size_t)n * kw, nrhox)) return fail(ctx, ATLASGPU_ENONFINITE, "%s: non-finite BHYD", name);
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t nt = (size_t)numnu * kw;
  const int nparts = h2 ? 14 : (helium ? 11 : 7);
  double *d_ws, *d_in, *d_dep, *d_out, *d_parts = nullptr;
  int r;
  // inputs: T, XNE, RHO, XNFP1, XNFP2, BMIN [kw], BHYD [6][kw], XNFP3..5, XNF4, XNF3 [kw]
  const size_t ndep = (size_t)(6 + 2 * kHLev + 9 + 10 + 24 + 3 + 14) * kw;
  if ((r = bufT(ctx, "kp_ws", numnu, &d_ws)) || (r = bufT(ctx, "kp_in", (size_t)17 * kw, &d_in)) ||
      (r = bufT(ctx, "kp_dep", ndep, &d_dep)) || (r = bufT(ctx, "kp_out", 3 * nt, &d_out)) ||
      (parts && (r = bufT(ctx, "kp_parts", (size_t)nparts * nt, &d_parts))))
    return r;
  CK(cudaMemsetAsync(d_in, 0, (size_t)17 * kw * sizeof(double), s));
  CK(cudaMemcpyAsync(d_ws, waveset, numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  const double* src[5] = {pp.t, pp.xne, pp.rho, pp.xnfp_h1, pp.xnfp_h2};
  for (int q = 0; q < 5; ++q)
    CK(cudaMemcpyAsync(d_in + (size_t)q * kw, src[q], nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  if (pp.bmin) CK(cudaMemcpyAsync(d_in + (size_t)5 * kw, pp.bmin, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  if (pp.bhyd)
    CK(cudaMemcpyAsync(d_in + (size_t)6 * kw, pp.bhyd, (size_t)6 * kw * sizeof(double), cudaMemcpyHostToDevice, s));
  if (helium) {
    const double* hsrc[4] = {pp.xnfp_he1, pp.xnfp_he2, pp.xnfp_he3, pp.xnf_he2};
    for (int q = 0; q < 4; ++q)
      CK(cudaMemcpyAsync(d_in + (size_t)(12 + q) * kw, hsrc[q], nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  if (h2) CK(cudaMemcpyAsync(d_in + (size_t)16 * kw, pp.xnf_he1, nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(d_out, 0, 3 * nt * sizeof(double), s));
  if (d_parts) CK(cudaMemsetAsync(d_parts, 0, (size_t)nparts * nt * sizeof(double), s));
  KappArgs a{};
  a.tb = (const KappDev*)ctx->bufs["kapp_tab"].first;
  a.numnu = numnu;
  a.nrhox = nrhox;
  a.kw = kw;
  a.waveset = d_ws;
  a.t = d_in;
  a.xne = d_in + kw;
  a.rho = d_in + 2 * kw;
  a.xnfp1 = d_in + 3 * kw;
  a.xnfp2 = d_in + 4 * kw;
  a.bmin = pp.bmin ? d_in + 5 * kw : nullptr;
  a.bhyd = pp.bhyd ? d_in + 6 * kw : nullptr;
  if (helium) {
    a.xnfp3 = d_in + 12 * kw;
    a.xnfp4 = d_in + 13 * kw;
    a.xnfp5 = d_in + 14 * kw;
    a.xnf4 = d_in + 15 * kw;
  }
  if (h2) {
    a.xnf3 = d_in + 16 * kw;
    a.h2 = (const KappH2Dev*)ctx->bufs["kapp_h2_tab"].first;
  }
  double* p = d_dep;
  double** dv[6] = {&a.d.hkt, &a.d.hckt, &a.d.tkev, &a.d.tlog, &a.d.theta, &a.d.xhmin};
  for (int q = 0; q < 6; ++q) {
    *dv[q] = p;
    p += kw;
  }
  a.d.w = p;
  p += (size_t)kHLev * kw;
  a.d.bz = p;
  p += (size_t)kHLev * kw;
  a.d.bp = p;
  p += (size_t)9 * kw;
  a.d.he_bolt = p;
  p += (size_t)10 * kw;
  a.d.he_boltn = p;
  p += (size_t)24 * kw;
  a.d.he_freet = p;
  a.d.he_boltex = p + kw;
  a.d.he_exlim = p + 2 * kw;
  p += (size_t)3 * kw;
  a.d.xnh2m = p;
  a.d.xnh2 = p + kw;
  a.d.ciaden = p + 2 * kw;
  a.d.ciait = p + 6 * kw;
  a.d.ciawt = p + 10 * kw;
  a.acont = d_out;
  a.sigmac = d_out + nt;
  a.scont = d_out + 2 * nt;
  a.parts = d_parts;
  a.nparts = nparts;
  {
    Timer tm(ctx, name);
    k_kapp_depth<<<(nrhox + 127) / 128, 128, 0, s>>>(a);
    CKL(ctx);
    const int blocks = std::min((numnu + kKappWarps - 1) / kKappWarps, ctx->nsm * 8);
    if (h2)
      k_kapp_nu<true, true><<<blocks, kKappWarps * 32, 0, s>>>(a);
    else if (helium)
      k_kapp_nu<true, false><<<blocks, kKappWarps * 32, 0, s>>>(a);
    else
      k_kapp_nu<false, false><<<blocks, kKappWarps * 32, 0, s>>>(a);
    CKL(ctx);
  }
  CK(cudaMemcpyAsync(acont, a.acont, nt * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(sigmac, a.sigmac, nt * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(scont, a.scont, nt * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (parts) CK(cudaMemcpyAsync(parts, d_parts, (size_t)nparts * nt * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

}  // namespace

extern "C" {

int atlasgpu_atlas_kapp_hydrogen(atlasgpu_ctx* ctx, int numnu, const double* waveset, int nrhox, int kw,
                                 const double* t, const double* xne, const double* rho, const double* xnfp1,
                                 const double* xnfp2, const double* bhyd, const double* bmin, double* acont,
                                 double* sigmac, double* scont, double* parts) {
  atlasgpu_kapp_pops pp{};
  pp.t = t;
  pp.xne = xne;
  pp.rho = rho;
  pp.xnfp_h1 = xnfp1;
  pp.xnfp_h2 = xnfp2;
  pp.bhyd = bhyd;
  pp.bmin = bmin;
  return kapp_run(ctx, "kapp_hydrogen", numnu, waveset, nrhox, kw, pp, false, acont, sigmac, scont, parts);
}

int atlasgpu_atlas_kapp(atlasgpu_ctx* ctx, int numnu, const double* waveset, int nrhox, int kw,
                        const atlasgpu_kapp_pops* pops, double* acont, double* sigmac, double* scont, double* parts) {
  if (!pops) return fail(ctx, ATLASGPU_EINVAL, "kapp: null populations");
  return kapp_run(ctx, "kapp", numnu, waveset, nrhox, kw, *pops, true, acont, sigmac, scont, parts);
}

int atlasgpu_atlas_set_stehle_tables(atlasgpu_ctx* ctx, const atlasgpu_stehle_series* stehle) {
  if (!ctx) return ATLASGPU_EINVAL;
  StehleDev* d;
  int r = stehle_upload(ctx, stehle, "ak_stehle", "atlas_set_stehle_tables", &d);
  if (r) return r;
  ctx->atlas_stehle = stehle != nullptr;
  return 0;
}

int atlasgpu_atlas_hlinop(atlasgpu_ctx* ctx, int numnu, const double* waveset, int nrhox, int kw, const double* t,
                          const double* xne, const double* rho, const double* xnfp1, const double* bhyd,
                          double* ahline, double* shline) {
  if (!ctx) return ATLASGPU_EINVAL;
  if (!ctx->kapp_set) return fail(ctx, ATLASGPU_ESTATE, "hlinop: tables not set");
  if (numnu < 1 || nrhox < 1 || kw < nrhox || !waveset || !t || !xne || !rho || !xnfp1 || !ahline || !shline)
    return fail(ctx, ATLASGPU_EINVAL, "hlinop: bad argument (numnu %d, nrhox %d, kw %d)", numnu, nrhox, kw);
  for (int i = 0; i < numnu; ++i)
    if (!(waveset[i] > 0.0) || !std::isfinite(waveset[i]))
      return fail(ctx, ATLASGPU_EINVAL, "hlinop: WAVESET(%d) = %g", i + 1, waveset[i]);
  if (!finite_all(t, nrhox) || !finite_all(xne, nrhox) || !finite_all(rho, nrhox) || !finite_all(xnfp1, nrhox))
    return fail(ctx, ATLASGPU_ENONFINITE, "hlinop: non-finite depth vector");
  for (int j = 0; j < nrhox; ++j)
    if (!(t[j] > 0.0) || !(rho[j] > 0.0) || !(xne[j] > 0.0))
      return fail(ctx, ATLASGPU_EINVAL, "hlinop: T, RHO or XNE not positive at depth %d", j + 1);
  if (bhyd)
    for (int n = 0; n < 6; ++n)
      for (int j = 0; j < nrhox; ++j)
        if (!std::isfinite(bhyd[(size_t)n * kw + j]) || !(bhyd[(size_t)n * kw + j] > 0.0))
          return fail(ctx, ATLASGPU_EINVAL, "hlinop: BHYD(%d, %d) not positive", j + 1, n + 1);
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t nt = (size_t)numnu * kw;
  double *d_ws, *d_in, *d_dep, *d_out;
  int r;
  const size_t ndep = (size_t)(6 + 2 * kHLev + 9) * kw;
  if ((r = bufT(ctx, "kp_ws", numnu, &d_ws)) || (r = bufT(ctx, "hl_in", (size_t)12 * kw, &d_in)) ||
      (r = bufT(ctx, "hl_dep", ndep, &d_dep)) || (r = bufT(ctx, "hl_out", 2 * nt, &d_out)))
    return r;
  CK(cudaMemsetAsync(d_in, 0, (size_t)12 * kw * sizeof(double), s));
  CK(cudaMemsetAsync(d_out, 0, 2 * nt * sizeof(double), s));
  CK(cudaMemcpyAsync(d_ws, waveset, numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  const double* src[4] = {t, xne, rho, xnfp1};
  for (int q = 0; q < 4; ++q)
    CK(cudaMemcpyAsync(d_in + (size_t)q * kw, src[q], nrhox * sizeof(double), cudaMemcpyHostToDevice, s));
  // XNFP(J,2) is not read by HLINOP; its slot stays zero
  if (bhyd) CK(cudaMemcpyAsync(d_in + (size_t)6 * kw, bhyd, (size_t)6 * kw * sizeof(double), cudaMemcpyHostToDevice, s));
  KappArgs a{};
  a.tb = (const KappDev*)ctx->bufs["kapp_tab"].first;
  a.numnu = numnu;
  a.nrhox = nrhox;
  a.kw = kw;
  a.waveset = d_ws;
  a.t = d_in;
  a.xne = d_in + kw;
  a.rho = d_in + 2 * kw;
  a.xnfp1 = d_in + 3 * kw;
  a.xnfp2 = d_in + 4 * kw;
  a.bhyd = bhyd ? d_in + 6 * kw : nullptr;
  double* p = d_dep;
  double** dv[6] = {&a.d.hkt, &a.d.hckt, &a.d.tkev, &a.d.tlog, &a.d.theta, &a.d.xhmin};
  for (int q = 0; q < 6; ++q) {
    *dv[q] = p;
    p += kw;
  }
  a.d.w = p;
  p += (size_t)kHLev * kw;
  a.d.bz = p;
  p += (size_t)kHLev * kw;
  a.d.bp = p;
  a.ahline = d_out;
  a.shline = d_out + nt;
  a.stehle = ctx->atlas_stehle ? (const StehleDev*)ctx->bufs["ak_stehle"].first : nullptr;
  {
    Timer tm(ctx, "hlinop");
    k_kapp_depth<<<(nrhox + 127) / 128, 128, 0, s>>>(a);
    CKL(ctx);
    const int blocks = std::min((numnu + kKappWarps - 1) / kKappWarps, ctx->nsm * 8);
    k_hlinop<<<blocks, kKappWarps * 32, 0, s>>>(a);
    CKL(ctx);
  }
  CK(cudaMemcpyAsync(ahline, a.ahline, nt * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(shline, a.shline, nt * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

}  // extern "C"
