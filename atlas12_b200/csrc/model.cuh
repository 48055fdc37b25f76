// model.cuh -- per-iteration steps of the device-resident ATLAS12 model that
// are not hot-path kernels of their own: hydrostatics and the surrogate
// EOS, KAPCONT's cutoff table, and the surrogate KAPP table of the RT pass.
// Shared by the single-model runtime (api_model.cu) and the batched one
// (api_batch.cu), whose kernels differ only in how they find a model.
#pragma once
#include "atlas.cuh"
#include "surrogate.cuh"
#include "tcorr.cuh"

namespace atlasgpu {

constexpr int kNState = 17;        // ModelState vectors
constexpr int kRossMax = 80 * 60;  // ROSSTAB_MAXTAB = kw*60 with the reference's kw = 80

// hydrostatics (iteration > 1), surrogate EOS / populations, Planck factors
// at depth j (0-based) of iteration `iter` (1-based)
__device__ inline void model_eos_depth(ModelState* ms, int iter, int j, int kw, double grav, double vturb_cms,
                                       double mh, double* xnfdop, double* dopple, double* xne_eos, double* txnxn,
                                       double* hkt, double* hckt, double* rho, ContCoef* cc) {
  const double t = ms->t[j];
  double p = ms->p[j];
  if (iter > 1) {
    // P = GRAV*RHOX - PRAD - PTURB - PCON (atlas12c.f90:513-519), PCON = 0
    p = grav * ms->rhox[j] - ms->prad[j] - ms->pturb[j] - 0.0;
    if (p <= 0.0) p = fmax(grav * ms->rhox[j] * 1.0e-4, 1.0e-10);
    ms->p[j] = p;
  }
  ContCoef c;
  const EosOut e = surrogate_depth(t, p, vturb_cms, mh, j, kw, xnfdop, dopple, &c);
  cc[j] = c;
  xne_eos[j] = e.xne;
  ms->xne[j] = e.xne;
  rho[j] = e.rho;
  const double tk = kKbol * t;
  hkt[j] = kHplanck / tk;
  hckt[j] = hkt[j] * kClight;
  // TXNXN = (XNF(H I) + 0.42 XNF(He I) + 0.85 XNF(H2)) (T/1e4)^0.3
  txnxn[j] = (e.nh * (1.0 - e.xh) + 0.42 * 0.085 * e.nh) * pow(t / 10000.0, 0.3);
}

// KAPCONT (atlas12_modules.f90:19072-19138) on the surrogate continuum: row
// nu (0-based) of TABCONT, threads over depths
__device__ inline void model_kapcont_row(int nu, const double* cutwave, int nwave, const double* waveset, int nrhox,
                                         int kw, const double* hkt, const ContCoef* cc, double* tabcont) {
  const double wave = cutwave[nu];
  const double freq = kClightNms / wave;
  for (int j = threadIdx.x; j < nrhox; j += blockDim.x) {
    double acont = 1.0e10, sigmac = 0.0;
    if (wave > waveset[0]) surrogate_kapp(cc[j], wave, acont, sigmac);
    const double stim = 1.0 - exp(-freq * hkt[j]);
    const double v = (acont + sigmac) * kLineCutoff / stim;
    tabcont[(size_t)nu * kw + j] = v;
    if (nu == nwave - 1) tabcont[(size_t)nwave * kw + j] = v;
  }
}

// KAPP stand-in for the RT pass: ACONT, SIGMAC [numnu][kw] from the surrogate
// continuum coefficients of this iteration's structure (grid-stride over
// blockIdx.x); xl, when given, is cleared over the same [numnu][kw] range
__device__ inline void model_kapp_range(const double* waveset, int numnu, int nrhox, int kw, const ContCoef* cc,
                                        double* acont, double* sigmac, double* xl) {
  const int64_t n = (int64_t)numnu * nrhox;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int nu = (int)(e / nrhox), j = (int)(e % nrhox);
    double ka, sg;
    surrogate_kapp(cc[j], waveset[nu], ka, sg);
    acont[(size_t)nu * kw + j] = ka;
    sigmac[(size_t)nu * kw + j] = sg;
    if (xl) xl[(size_t)nu * kw + j] = 0.0;
  }
}

}  // namespace atlasgpu
