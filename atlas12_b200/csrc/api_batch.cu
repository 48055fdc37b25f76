// api_batch.cu -- many ATLAS12 atmospheres iterated together on one device.
//
// The reference runs one model per process and grids of models as SLURM
// arrays of single-core jobs (scripts/runat12_grid.slurm:1-16); each process
// runs the iteration loop of atlas12c.f90:496-606.  Here a batch holds
// `nslots` atmospheres that share one frequency grid, one line list and the
// Voigt tables; each slot has its own parameters, structure, populations,
// opacities and ROSSTAB history.  One captured CUDA graph runs one iteration
// of every RUNNING slot (seven launches for the whole batch, model index in
// the grid's y or x dimension).  A slot's own status word, written by the
// finish kernel, takes it out of the iteration when it converges, when
// max |FLXERR| stops being finite, or at its iteration cap, so the graph can
// be replayed many times between host polls, and a finished slot can be
// loaded with the next model (a work queue) while the others keep going.
#include <algorithm>
#include <cmath>
#include <vector>

#include "api_common.cuh"
#include "model.cuh"

using namespace atlasgpu;

namespace {

constexpr int kHist = ATLASGPU_BATCH_MAX_ITER;  // max |FLXERR| history per slot

struct BatchCtl {
  int status;  // ATLASGPU_SLOT_*
  int iter;    // iterations completed
  int max_iter;
  int pad;
  double tol;     // percent; <= 0: run to max_iter
  double maxerr;  // last max |FLXERR| (percent)
  double teff, grav, vturb_cms, mh;
};

// base pointers of the per-slot arrays (slot b's part at b * per-slot size)
struct BatchDev {
  BatchCtl* ctl;
  ModelState* ms;
  RossStore* R;
  double *xnfdop, *dopple;                     // [B][nspec][kw]
  double *xne_eos, *txnxn, *hkt, *hckt, *rho;  // [B][kw]
  ContCoef* cc;                                // [B][kw]
  double *acont, *sigmac, *xl;                 // [B][numnu][kw]
  unsigned long long* xfix;                    // [B][numnu][3][kw] LINOP1's exact sums
  double *fscale, *funscale;                   // [B][kw] their per-depth scale
  const double* cgfmax;                        // [nspec] largest CGF per species (shared line list)
  double* tabcont;                             // [B][nwave+1][kw]
  double* partial;                             // [B][nwl][kAcc*kw+1]
  double* rt_rec;                              // [B][numnu][rt_rec_stride(kw)] split RT pass records
  double* sum;                                 // [B][kAcc*kw+1]
  double* hist;                                // [B][kHist]
  double* hsurf;                               // [B][numnu] HNU(1) of the last iteration
  const double *waveset, *cutwave;
  int numnu, nwave, nrhox, kw, nspec, nwl;
};

__device__ __forceinline__ bool running(const BatchCtl* ctl, int b) { return ctl[b].status == ATLASGPU_SLOT_RUNNING; }

__global__ void k_batch_eos(BatchDev d) {
  const int b = blockIdx.x, j = threadIdx.x;
  if (!running(d.ctl, b) || j >= d.nrhox) return;
  const BatchCtl c = d.ctl[b];
  const size_t o = (size_t)b * d.kw, os = (size_t)b * d.nspec * d.kw;
  model_eos_depth(d.ms + b, c.iter + 1, j, d.kw, c.grav, c.vturb_cms, c.mh, d.xnfdop + os, d.dopple + os,
                  d.xne_eos + o, d.txnxn + o, d.hkt + o, d.hckt + o, d.rho + o, d.cc + o);
  fix_scale_depth(d.xnfdop + os, d.nspec, d.kw, j, d.cgfmax, d.fscale + o, d.funscale + o);
}

// XLINES of every running slot from its fixed-point sums
__global__ void k_batch_fixfin(BatchDev d) {
  const int b = blockIdx.y;
  if (!running(d.ctl, b)) return;
  const size_t on = (size_t)b * d.numnu * d.kw;
  fix_finalize_range(d.xfix + kFixWords * on, d.funscale + (size_t)b * d.kw, d.numnu, d.nrhox, d.kw, d.xl + on);
}

// KAPCONT on a slot's first iteration only (atlas12c.f90:562)
__global__ void k_batch_kapcont(BatchDev d) {
  const int b = blockIdx.y;
  if (!running(d.ctl, b) || d.ctl[b].iter != 0) return;
  const size_t o = (size_t)b * d.kw;
  model_kapcont_row(blockIdx.x, d.cutwave, d.nwave, d.waveset, d.nrhox, d.kw, d.hkt + o, d.cc + o,
                    d.tabcont + (size_t)b * (d.nwave + 1) * d.kw);
}

__global__ void k_batch_kapp(BatchDev d) {
  const int b = blockIdx.y;
  if (!running(d.ctl, b)) return;
  const size_t o = (size_t)b * d.numnu * d.kw;
  model_kapp_range(d.waveset, d.numnu, d.nrhox, d.kw, d.cc + (size_t)b * d.kw, d.acont + o, d.sigmac + o, d.xl + o);
}

// LINOP1 per running slot (blockIdx.y): the slot's grid-stride share of the
// line list.  (One work queue over all running slots, CTAs taking 256-line
// entries, measured 5 % slower on the bench's 32-slot batch: 2.39 against
// 2.27 ms per model-iteration.)
// kDry: the counting pass of a timed iteration (the same walks, no adds)
template <bool F32, bool kDry = false>
__global__ void __launch_bounds__(256, kLinopMinBlocks) k_batch_linop(const LinopArgs* __restrict__ args, const BatchCtl* ctl,
                                                                      unsigned long long* work) {
  const int b = blockIdx.y;
  if (!running(ctl, b)) return;
  LinopArgs a = args[b];
  a.work = work;
  linop_body<F32, kDry>(a);
}

// the split RT pass (k_rt_pre / k_rt_solve / k_rt_post bodies) per running slot
__global__ void __launch_bounds__(kRtSplitWarps * 32, 6) k_batch_rt_pre(const RtArgs* __restrict__ args,
                                                                       const BatchCtl* ctl) {
  const int b = blockIdx.y;
  if (!running(ctl, b)) return;
  rt_pre_body(args[b]);
}
__global__ void __launch_bounds__(kRtSolveThreads, kRtSolveMinBlocks) k_batch_rt_solve(const RtArgs* __restrict__ args,
                                                                                    const BatchCtl* ctl,
                                                                                    unsigned long long* work) {
  const int b = blockIdx.y;
  if (!running(ctl, b)) return;
  RtArgs a = args[b];
  a.work = work;
  rt_solve_body(a);
}
__global__ void __launch_bounds__(kRtSolveThreads, kRtSeriesMinBlocks) k_batch_rt_series(const RtArgs* __restrict__ args,
                                                                                      const BatchCtl* ctl,
                                                                                      unsigned long long* work) {
  const int b = blockIdx.y;
  if (!running(ctl, b)) return;
  RtArgs a = args[b];
  a.work = work;
  rt_series_body(a);
}
__global__ void __launch_bounds__(kRtSplitWarps * 32, 4) k_batch_rt_post(const RtArgs* __restrict__ args,
                                                                        const BatchCtl* ctl) {
  const int b = blockIdx.y;
  if (!running(ctl, b)) return;
  RtArgs a = args[b];
  a.teff = ctl[b].teff;
  rt_post_body(a);
}

__global__ void __launch_bounds__(kRedCols* kRedRows) k_batch_reduce(BatchDev d) {
  const int b = blockIdx.y;
  if (!running(d.ctl, b)) return;
  const size_t stride = (size_t)kAcc * d.kw + 1;
  reduce_body(d.partial + (size_t)b * d.nwl * stride, d.nwl, d.kw, d.sum + (size_t)b * stride);
}

__global__ void __launch_bounds__(kFinThreads) k_batch_finish(BatchDev d) {
  extern __shared__ __align__(16) double fin_smem[];
  const int b = blockIdx.x;
  if (!running(d.ctl, b)) return;
  const BatchCtl c = d.ctl[b];
  __syncthreads();  // every thread has read the slot's control word before thread 0 rewrites it
  const double e = b_atlas_finish(d.ms + b, d.sum + (size_t)b * (kAcc * d.kw + 1), d.kw, d.nrhox, c.iter + 1,
                                  c.teff, c.grav, d.R + b, fin_smem);
  if (threadIdx.x == 0) {
    const int it = c.iter + 1;
    BatchCtl& w = d.ctl[b];
    w.maxerr = e;
    w.iter = it;
    if (it <= kHist) d.hist[(size_t)b * kHist + it - 1] = e;
    if (!(e == e)) w.status = ATLASGPU_SLOT_NONFINITE;
    else if (c.tol > 0.0 && e <= c.tol) w.status = ATLASGPU_SLOT_CONVERGED;
    else if (it >= c.max_iter) w.status = ATLASGPU_SLOT_CAPPED;
  }
}

template <class T>
int balloc(atlasgpu_ctx* ctx, T** p, size_t n) {
  if (cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(ctx, ATLASGPU_ENOMEM, "batch: cudaMalloc of %zu bytes", n * sizeof(T));
  }
  return 0;
}

}  // namespace

struct atlasgpu_batch {
  int nslots = 0, nrhox = 0, kw = 0, numnu = 0, nwave = 0, nspec = kSurrNspec;
  int64_t nlines = 0;
  BatchDev d{};
  // batch-wide device data
  double *waveset = nullptr, *rcoset = nullptr, *cutwave = nullptr, *h0 = nullptr, *h1 = nullptr, *h2 = nullptr;
  float4* hf = nullptr;
  int graph_precision = -1;  // precision the captured graph was built with
  double *ross = nullptr, *state = nullptr;
  int32_t *iwavetab = nullptr, *linedata = nullptr;
  AtlasLine* lines = nullptr;
  LinopArgs* la = nullptr;
  RtArgs* ra = nullptr;
  unsigned long long* cnt = nullptr;
  int grid_linop = 1, grid_kapp = 1;
  RtSplitShape rt_sh;                         // launch shape of the split RT pass
  int linop_ctas_per_sm = 16, rt_waves = 32;  // launch shape (atlasgpu_batch_set_shape)
  size_t partial_rows = 0;                    // allocated partial-sum rows per slot
  std::vector<RtArgs> ra_host;                // per-slot RT arguments (rebuilt with the shape)
  size_t smem_fin = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
};

namespace {

int enqueue_batch(atlasgpu_ctx* ctx, atlasgpu_batch* B, bool timed) {
  cudaStream_t s = ctx->stream;
  const bool was = ctx->timing;
  ctx->timing = was && timed;
  const int nb = B->nslots;
  {
    Timer tm(ctx, "batch_eos");
    k_batch_eos<<<nb, 128, 0, s>>>(B->d);
    CKL(ctx);
  }
  {
    Timer tm(ctx, "batch_kapcont");
    k_batch_kapcont<<<dim3(B->nwave, nb), 128, 0, s>>>(B->d);
    CKL(ctx);
  }
  {
    Timer tm(ctx, "batch_kapp");
    k_batch_kapp<<<dim3(B->grid_kapp, nb), 256, 0, s>>>(B->d);
    CKL(ctx);
  }
  if (B->nlines > 0) {
    if (ctx->timing) {
      // the atomics the exact sums issue, counted by a pass that walks the
      // same wings and adds nothing (the numerator of LINOP1's roofline; the
      // timed launch below carries no counting)
      unsigned long long* dry;
      if (bufT(ctx, "linop_dry_cnt", 2, &dry) == 0 &&
          cudaMemsetAsync(dry, 0, 2 * sizeof(unsigned long long), s) == cudaSuccess) {
        if (ctx->precision == ATLASGPU_PREC_MIXED)
          k_batch_linop<true, true><<<dim3(B->grid_linop, nb), 256, 0, s>>>(B->la, B->d.ctl, dry);
        else
          k_batch_linop<false, true><<<dim3(B->grid_linop, nb), 256, 0, s>>>(B->la, B->d.ctl, dry);
        CKL(ctx);
        unsigned long long h[2] = {0, 0};
        CK(cudaMemcpyAsync(h, dry, sizeof h, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        ctx->kwork["batch_linop_atomics"] = (double)h[1];
      }
    }
    unsigned long long* work = work_counters(ctx, 1);
    {
      Timer tm(ctx, "batch_linop");
      if (ctx->precision == ATLASGPU_PREC_MIXED)
        k_batch_linop<true><<<dim3(B->grid_linop, nb), 256, 0, s>>>(B->la, B->d.ctl, work);
      else
        k_batch_linop<false><<<dim3(B->grid_linop, nb), 256, 0, s>>>(B->la, B->d.ctl, work);
      CKL(ctx);
    }
    work_collect(ctx, work, {"batch_linop_points"});
    {
      Timer tm(ctx, "batch_fixfin");
      k_batch_fixfin<<<dim3(B->grid_kapp, nb), 256, 0, s>>>(B->d);
      CKL(ctx);
    }
  }
  {
    Timer tm(ctx, "batch_rt");
    const RtSplitShape& sh = B->rt_sh;
    {
      Timer t1(ctx, "batch_rt_pre");
      k_batch_rt_pre<<<dim3(sh.pre_blocks, nb), kRtSplitWarps * 32, rt_pre_smem_bytes(), s>>>(B->ra, B->d.ctl);
      CKL(ctx);
    }
    {
      unsigned long long* work = work_counters(ctx, 3);
      {
        Timer t2(ctx, "batch_rt_solve");
        k_batch_rt_series<<<dim3(sh.solve_blocks, nb), kRtSolveThreads, 0, s>>>(B->ra, B->d.ctl, work);
        CKL(ctx);
        k_batch_rt_solve<<<dim3(sh.solve_blocks, nb), kRtSolveThreads, rt_solve_smem_bytes(), s>>>(B->ra,
                                                                                                 B->d.ctl, work);
        CKL(ctx);
      }
      work_collect(ctx, work, {"batch_rt_eliminated", "batch_rt_series", "batch_rt_series_steps"});
    }
    {
      Timer t3(ctx, "batch_rt_post");
      k_batch_rt_post<<<dim3(sh.post_blocks, nb), kRtSplitWarps * 32, rt_post_smem_bytes(B->nrhox), s>>>(
          B->ra, B->d.ctl);
      CKL(ctx);
    }
  }
  {
    Timer tm(ctx, "batch_reduce");
    const int stride = kAcc * B->kw + 1;
    k_batch_reduce<<<dim3((stride + kRedCols - 1) / kRedCols, nb), dim3(kRedCols, kRedRows), 0, s>>>(B->d);
    CKL(ctx);
  }
  {
    Timer tm(ctx, "batch_finish");
    k_batch_finish<<<nb, kFinThreads, B->smem_fin, s>>>(B->d);
    CKL(ctx);
  }
  ctx->timing = was;
  return 0;
}

// Launch shape: LINOP1 CTAs per SM over the whole batch, and the split RT
// pass's warps and pair groups sized for about rt_waves resident waves over
// the batch (each takes a contiguous run of one slot's frequencies).  Grows
// the partial-sum buffer when a shape needs more rows, rewrites the per-slot
// RT arguments and drops the captured graph.
int apply_shape(atlasgpu_ctx* ctx, atlasgpu_batch* B, int linop_ctas_per_sm, int rt_waves) {
  const int nb = B->nslots;
  const size_t stride = (size_t)kAcc * B->kw + 1;
  const RtSplitShape sh = rt_split_shape(B->numnu, ctx->nsm, nb, rt_waves);
  const size_t rows = (size_t)sh.rows();
  CK(cudaStreamSynchronize(ctx->stream));
  if (rows > B->partial_rows) {
    if (B->d.partial) cudaFree(B->d.partial);
    B->d.partial = nullptr;
    if (cudaMalloc((void**)&B->d.partial, (size_t)nb * rows * stride * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      B->partial_rows = 0;
      return fail(ctx, ATLASGPU_ENOMEM, "batch: partial sums for %zu groups per slot", rows);
    }
    B->partial_rows = rows;
  }
  B->rt_sh = sh;
  B->d.nwl = (int)rows;
  B->grid_linop = std::max(1, ctx->nsm * linop_ctas_per_sm / nb);
  B->linop_ctas_per_sm = linop_ctas_per_sm;
  B->rt_waves = rt_waves;
  for (int b = 0; b < nb; ++b) {
    rt_split_args(B->ra_host[b], sh);
    B->ra_host[b].partial = B->d.partial + (size_t)b * rows * stride;
  }
  CK(cudaMemcpy(B->ra, B->ra_host.data(), nb * sizeof(RtArgs), cudaMemcpyHostToDevice));
  if (B->gexec) cudaGraphExecDestroy(B->gexec);
  if (B->graph) cudaGraphDestroy(B->graph);
  B->gexec = nullptr;
  B->graph = nullptr;
  return 0;
}

}  // namespace

extern "C" {

int atlasgpu_batch_destroy(atlasgpu_ctx* ctx, atlasgpu_batch* B) {
  if (!B) return ATLASGPU_EINVAL;
  if (ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
  }
  if (B->gexec) cudaGraphExecDestroy(B->gexec);
  if (B->graph) cudaGraphDestroy(B->graph);
  const BatchDev& d = B->d;
  void* ps[] = {d.xfix, d.fscale, d.funscale, (void*)d.cgfmax,
                d.ctl, d.ms, d.R, d.xnfdop, d.dopple, d.xne_eos, d.txnxn, d.hkt, d.hckt, d.rho, d.cc, d.acont,
                d.sigmac, d.xl, d.tabcont, d.partial, d.rt_rec, d.sum, d.hist, d.hsurf, B->waveset, B->rcoset, B->cutwave, B->h0,
                B->h1, B->h2, B->hf, B->ross, B->state, B->iwavetab, B->linedata, B->lines, B->la, B->ra, B->cnt};
  for (void* p : ps)
    if (p) cudaFree(p);
  delete B;
  return ATLASGPU_OK;
}

int atlasgpu_batch_create(atlasgpu_ctx* ctx, const atlasgpu_model_desc* dsc, int nslots, atlasgpu_batch** out) {
  if (!ctx || !dsc || !out) return fail(ctx, ATLASGPU_EINVAL, "batch_create: null argument");
  *out = nullptr;
  if (!ctx->ops_set) return fail(ctx, ATLASGPU_ESTATE, "batch_create: operators not set");
  if (nslots < 1 || nslots > ATLASGPU_BATCH_MAX_SLOTS || dsc->nrhox < 16 || dsc->nrhox > kKwMax ||
      dsc->numnu < 2 || dsc->nwave < 1 || dsc->nlines < 0 || !dsc->waveset || !dsc->rcoset || !dsc->cutoff_wave ||
      (dsc->nlines > 0 && !dsc->linedata) || !dsc->h0tab || !dsc->h1tab || !dsc->h2tab)
    return fail(ctx, ATLASGPU_EINVAL, "batch_create: bad descriptor or slot count %d", nslots);
  for (int i = 1; i < dsc->numnu; ++i)
    if (!(dsc->waveset[i] > dsc->waveset[i - 1])) return fail(ctx, ATLASGPU_EINVAL, "WAVESET not increasing");
  for (int i = 1; i < dsc->nwave; ++i)
    if (!(dsc->cutoff_wave[i] > dsc->cutoff_wave[i - 1]))
      return fail(ctx, ATLASGPU_EINVAL, "cutoff grid not increasing");
  cudaSetDevice(ctx->device);
  atlasgpu_batch* B = new atlasgpu_batch();
  B->nslots = nslots;
  B->nrhox = B->kw = dsc->nrhox;
  B->numnu = dsc->numnu;
  B->nwave = dsc->nwave;
  B->nlines = dsc->nlines;
  const int kw = B->kw, nb = nslots;
  const size_t stride = (size_t)kAcc * kw + 1;
  B->grid_kapp = std::max(1, ctx->nsm * 8 / nb);
  BatchDev& d = B->d;
  d.numnu = B->numnu;
  d.nwave = B->nwave;
  d.nrhox = B->nrhox;
  d.kw = kw;
  d.nspec = B->nspec;
  const size_t nsk = (size_t)B->nspec * kw, nnk = (size_t)B->numnu * kw;
  int r = 0;
  if ((r = balloc(ctx, &d.ctl, nb)) || (r = balloc(ctx, &d.ms, nb)) || (r = balloc(ctx, &d.R, nb)) ||
      (r = balloc(ctx, &d.xnfdop, nb * nsk)) || (r = balloc(ctx, &d.dopple, nb * nsk)) ||
      (r = balloc(ctx, &d.xne_eos, (size_t)nb * kw)) || (r = balloc(ctx, &d.txnxn, (size_t)nb * kw)) ||
      (r = balloc(ctx, &d.hkt, (size_t)nb * kw)) || (r = balloc(ctx, &d.hckt, (size_t)nb * kw)) ||
      (r = balloc(ctx, &d.rho, (size_t)nb * kw)) || (r = balloc(ctx, &d.cc, (size_t)nb * kw)) ||
      (r = balloc(ctx, &d.acont, nb * nnk)) || (r = balloc(ctx, &d.sigmac, nb * nnk)) ||
      (r = balloc(ctx, &d.xl, nb * nnk)) || (r = balloc(ctx, &d.tabcont, (size_t)nb * (B->nwave + 1) * kw)) ||
      (r = balloc(ctx, &d.sum, nb * stride)) || (r = balloc(ctx, &d.rt_rec, nb * (size_t)B->numnu * rt_rec_stride(kw))) ||
      (r = balloc(ctx, &d.hist, (size_t)nb * kHist)) || (r = balloc(ctx, &d.hsurf, nb * (size_t)B->numnu)) ||
      (r = balloc(ctx, &B->waveset, B->numnu)) ||
      (r = balloc(ctx, &B->rcoset, B->numnu)) || (r = balloc(ctx, &B->cutwave, B->nwave)) ||
      (r = balloc(ctx, &B->iwavetab, B->nwave + 1)) || (r = balloc(ctx, &B->h0, 2001)) ||
      (r = balloc(ctx, &B->h1, 2001)) || (r = balloc(ctx, &B->h2, 2001)) || (r = balloc(ctx, &B->hf, 2001)) ||
      (r = balloc(ctx, &B->ross, (size_t)nb * 3 * kRossMax)) || (r = balloc(ctx, &B->state, (size_t)nb * kNState * kw)) ||
      (r = balloc(ctx, &B->linedata, (size_t)B->nlines * 4)) || (r = balloc(ctx, &B->lines, (size_t)B->nlines)) ||
      (r = balloc(ctx, &B->la, nb)) || (r = balloc(ctx, &B->ra, nb)) || (r = balloc(ctx, &B->cnt, 2)) ||
      (r = balloc(ctx, &d.xfix, (size_t)kFixWords * nb * nnk)) || (r = balloc(ctx, &d.fscale, (size_t)nb * kw)) ||
      (r = balloc(ctx, &d.funscale, (size_t)nb * kw)) || (r = balloc(ctx, (double**)&d.cgfmax, (size_t)B->nspec))) {
    atlasgpu_batch_destroy(ctx, B);
    return r;
  }
  d.waveset = B->waveset;
  d.cutwave = B->cutwave;
  B->smem_fin = fin_smem_bytes(kw, kRossMax);
  if (B->smem_fin > (size_t)ctx->smem_optin) {
    atlasgpu_batch_destroy(ctx, B);
    return fail(ctx, ATLASGPU_EINVAL, "batch_create: finish needs %zu B of shared memory", B->smem_fin);
  }
  CK(cudaFuncSetAttribute(k_batch_rt_pre, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rt_pre_smem_bytes()));
  CK(cudaFuncSetAttribute(k_batch_rt_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rt_solve_smem_bytes()));
  CK(cudaFuncSetAttribute(k_batch_rt_post, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)rt_post_smem_bytes(B->nrhox)));
  CK(cudaFuncSetAttribute(k_batch_finish, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->smem_fin));
  cudaStream_t s = ctx->stream;
  // slots start idle; state pointers, ROSSTAB stores and per-slot kernel arguments are fixed for life
  std::vector<BatchCtl> ctl(nb);
  std::vector<ModelState> ms(nb);
  std::vector<RossStore> R(nb);
  std::vector<LinopArgs> la(nb);
  std::vector<RtArgs> ra(nb);
  for (int b = 0; b < nb; ++b) {
    ctl[b] = BatchCtl{ATLASGPU_SLOT_IDLE, 0, 0, 0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0};
    double* st = B->state + (size_t)b * kNState * kw;
    double** f[kNState] = {&ms[b].t, &ms[b].rhox, &ms[b].p, &ms[b].xne, &ms[b].abross, &ms[b].prad,
                           &ms[b].vturb, &ms[b].pturb, &ms[b].tauros, &ms[b].accrad, &ms[b].raden,
                           &ms[b].oldt1, &ms[b].flxerr, &ms[b].dtflux, &ms[b].dtlamb, &ms[b].dtsurf, &ms[b].t1};
    for (int q = 0; q < kNState; ++q) *f[q] = st + (size_t)q * kw;
    ms[b].pradk0 = 0.0;
    ms[b].maxerr = 0.0;
    double* rs = B->ross + (size_t)b * 3 * kRossMax;
    R[b] = RossStore{0, kRossMax, 0.0, 1.0, 0.0, 1.0, rs, rs + kRossMax, rs + 2 * kRossMax};
    const size_t o = (size_t)b * kw, os = (size_t)b * nsk, on = (size_t)b * nnk;
    la[b] = LinopArgs{B->lines, B->nlines, B->nrhox, kw, B->nspec, B->numnu, d.xnfdop + os, d.dopple + os,
                      d.xne_eos + o, d.txnxn + o, d.hckt + o, d.tabcont + (size_t)b * (B->nwave + 1) * kw,
                      B->waveset, B->h0, B->h1, B->h2, B->hf, d.xl + on, nullptr, B->cnt};
    la[b].xfix = d.xfix + kFixWords * on;
    la[b].fscale = d.fscale + o;
    ra[b] = RtArgs{ctx->ops, B->numnu, B->nrhox, kw, B->waveset, B->rcoset, d.acont + on, d.sigmac + on, nullptr,
                   d.xl + on, ms[b].rhox, ms[b].t, d.hkt + o, 0.0, 1, 1, kw, nullptr,
                   d.hsurf + (size_t)b * B->numnu, nullptr};
    ra[b].rec = d.rt_rec + (size_t)b * B->numnu * rt_rec_stride(kw);
  }
  B->ra_host = ra;
  CK(cudaMemcpyAsync(d.ctl, ctl.data(), nb * sizeof(BatchCtl), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d.ms, ms.data(), nb * sizeof(ModelState), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d.R, R.data(), nb * sizeof(RossStore), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(B->la, la.data(), nb * sizeof(LinopArgs), cudaMemcpyHostToDevice, s));

  CK(cudaMemsetAsync(B->state, 0, (size_t)nb * kNState * kw * sizeof(double), s));
  CK(cudaMemsetAsync(d.xnfdop, 0, nb * nsk * sizeof(double), s));
  {
    // dopple must be nonzero where a line may look: fill with 1 (the populations are 0 there)
    std::vector<double> one(nb * nsk, 1.0);
    CK(cudaMemcpy(d.dopple, one.data(), one.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  CK(cudaMemsetAsync(d.hist, 0, (size_t)nb * kHist * sizeof(double), s));
  CK(cudaMemcpyAsync(B->waveset, dsc->waveset, B->numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(B->rcoset, dsc->rcoset, B->numnu * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(B->cutwave, dsc->cutoff_wave, B->nwave * sizeof(double), cudaMemcpyHostToDevice, s));
  std::vector<int32_t> iwt(B->nwave + 1);
  const double RATIOLG = log(1.0 + 1.0 / 2000000.0);
  for (int i = 0; i < B->nwave; ++i) iwt[i] = (int32_t)(log(dsc->cutoff_wave[i]) / RATIOLG + 0.5);
  iwt[B->nwave] = 1 << 30;
  CK(cudaMemcpyAsync(B->iwavetab, iwt.data(), iwt.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (B->nlines > 0)
    CK(cudaMemcpyAsync(B->linedata, dsc->linedata, (size_t)B->nlines * 4 * sizeof(int32_t), cudaMemcpyHostToDevice,
                       s));
  CK(cudaMemcpyAsync(B->h0, dsc->h0tab, 2001 * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(B->h1, dsc->h1tab, 2001 * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(B->h2, dsc->h2tab, 2001 * sizeof(double), cudaMemcpyHostToDevice, s));
  {
    const std::vector<float4> hf = pack_voigt_f32(dsc->h0tab, dsc->h1tab, dsc->h2tab, 2001);
    CK(cudaMemcpy(B->hf, hf.data(), hf.size() * sizeof(float4), cudaMemcpyHostToDevice));
  }
  CK(cudaMemsetAsync(B->cnt, 0, 2 * sizeof(unsigned long long), s));
  double* tl;
  {
    const bool fresh = ctx->bufs.find("tablog") == ctx->bufs.end();
    if ((r = bufT(ctx, "tablog", 65536, &tl))) {
      atlasgpu_batch_destroy(ctx, B);
      return r;
    }
    if (fresh) {
      std::vector<double> ht(65536);
      for (int k = 0; k < 65536; ++k) ht[k] = pow(10.0, (double)((k - 32768) - 16384) * 0.001);
      CK(cudaMemcpy(tl, ht.data(), 65536 * sizeof(double), cudaMemcpyHostToDevice));
    }
  }
  if (B->nlines > 0 && (r = atlas_prep_lines(ctx, B->linedata, dsc->linedata, B->nlines, tl, B->waveset,
                                              dsc->waveset, B->numnu, B->iwavetab, B->nwave, B->nspec, B->lines))) {
    atlasgpu_batch_destroy(ctx, B);
    return r;
  }
  // exact XLINES sums: zeroed words, the largest CGF per species for the scales
  CK(cudaMemsetAsync(d.xfix, 0, (size_t)kFixWords * nb * nnk * sizeof(unsigned long long), s));
  CK(cudaMemsetAsync((void*)d.cgfmax, 0, (size_t)B->nspec * sizeof(double), s));
  if (B->nlines > 0) {
    k_cgf_max<<<grid_for(ctx, B->nlines, 256, 8), 256, 0, s>>>(B->lines, B->nlines, B->nspec,
                                                                (unsigned long long*)d.cgfmax);
    CKL(ctx);
  }
  CK(cudaStreamSynchronize(s));
  if ((r = apply_shape(ctx, B, B->linop_ctas_per_sm, B->rt_waves))) {
    atlasgpu_batch_destroy(ctx, B);
    return r;
  }
  *out = B;
  return 0;
}

int atlasgpu_batch_set_shape(atlasgpu_ctx* ctx, atlasgpu_batch* B, int linop_ctas_per_sm, int rt_waves) {
  if (!ctx || !B || linop_ctas_per_sm < 1 || linop_ctas_per_sm > 64 || rt_waves < 1 || rt_waves > 256)
    return fail(ctx, ATLASGPU_EINVAL, "batch_set_shape: linop CTAs per SM %d (1..64), RT waves %d (1..256)",
                linop_ctas_per_sm, rt_waves);
  cudaSetDevice(ctx->device);
  return apply_shape(ctx, B, linop_ctas_per_sm, rt_waves);
}

int atlasgpu_batch_get_shape(atlasgpu_ctx* ctx, atlasgpu_batch* B, int* linop_ctas_per_sm, int* rt_waves) {
  if (!ctx || !B) return fail(ctx, ATLASGPU_EINVAL, "batch_get_shape: null");
  if (linop_ctas_per_sm) *linop_ctas_per_sm = B->linop_ctas_per_sm;
  if (rt_waves) *rt_waves = B->rt_waves;
  return 0;
}

int atlasgpu_batch_load(atlasgpu_ctx* ctx, atlasgpu_batch* B, int slot, double teff, double logg, double vturb_kms,
                        double mh, const double* t, const double* p, const double* rhox, int max_iter,
                        double tol_percent) {
  if (!ctx || !B || slot < 0 || slot >= B->nslots || !t || !p || !rhox || !(teff > 0.0) || !(vturb_kms >= 0.0) ||
      max_iter < 1 || max_iter > kHist)
    return fail(ctx, ATLASGPU_EINVAL, "batch_load: bad argument (slot %d, max_iter %d)", slot, max_iter);
  for (int j = 0; j < B->nrhox; ++j)
    if (!(t[j] > 0.0) || !(p[j] > 0.0) || !(rhox[j] > 0.0))
      return fail(ctx, ATLASGPU_EINVAL, "batch_load: non-positive T, P or RHOX at depth %d", j + 1);
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const int kw = B->kw;
  // a fresh model: every state vector zero except T, RHOX, P, VTURB and TAUROS = TAUSTD
  std::vector<double> h((size_t)kNState * kw, 0.0);
  for (int j = 0; j < B->nrhox; ++j) {
    h[0 * kw + j] = t[j];
    h[1 * kw + j] = rhox[j];
    h[2 * kw + j] = p[j];
    h[6 * kw + j] = vturb_kms * 1.0e5;
    h[8 * kw + j] = pow(10.0, -6.875 + 0.125 * j);
  }
  ModelState ms;
  CK(cudaMemcpy(&ms, B->d.ms + slot, sizeof ms, cudaMemcpyDeviceToHost));
  ms.pradk0 = 0.0;
  ms.maxerr = 0.0;
  double* rs = B->ross + (size_t)slot * 3 * kRossMax;
  const RossStore R0{0, kRossMax, 0.0, 1.0, 0.0, 1.0, rs, rs + kRossMax, rs + 2 * kRossMax};
  const BatchCtl c{ATLASGPU_SLOT_RUNNING, 0, max_iter, 0, tol_percent, 0.0, teff, pow(10.0, logg),
                   vturb_kms * 1.0e5, mh};
  // pageable sources: each copy is complete when the call returns
  CK(cudaMemcpyAsync(B->state + (size_t)slot * kNState * kw, h.data(), h.size() * sizeof(double),
                     cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(B->d.ms + slot, &ms, sizeof ms, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(B->d.R + slot, &R0, sizeof R0, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(B->d.hist + (size_t)slot * kHist, 0, kHist * sizeof(double), s));
  CK(cudaMemcpyAsync(B->d.ctl + slot, &c, sizeof c, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int atlasgpu_batch_step(atlasgpu_ctx* ctx, atlasgpu_batch* B, int n) {
  if (!ctx || !B || n < 0) return fail(ctx, ATLASGPU_EINVAL, "batch_step: bad argument");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  int r;
  for (int i = 0; i < n; ++i) {
    if (ctx->timing) {
      // per-kernel CUDA-event timing needs the launches outside a graph
      if ((r = enqueue_batch(ctx, B, true))) return r;
      continue;
    }
    if (B->gexec && B->graph_precision != ctx->precision) {
      // the graph holds the kernels of the precision it was captured with
      cudaGraphExecDestroy(B->gexec);
      cudaGraphDestroy(B->graph);
      B->gexec = nullptr;
      B->graph = nullptr;
    }
    if (!B->gexec) {
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const int64_t l0 = ctx->launches;
      r = enqueue_batch(ctx, B, false);
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(s, &g);
      if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
      }
      if (ec != cudaSuccess) return fail(ctx, ATLASGPU_ECUDA, "batch graph capture: %s", cudaGetErrorString(ec));
      B->graph = g;
      CK(cudaGraphInstantiate(&B->gexec, g, 0));
      B->graph_precision = ctx->precision;
      ctx->launches = l0;  // counted when replayed
    }
    CK(cudaGraphLaunch(B->gexec, s));
    ctx->launches += B->nlines > 0 ? 8 : 6;
  }
  return 0;
}

int atlasgpu_batch_poll(atlasgpu_ctx* ctx, atlasgpu_batch* B, int* status, int* iters, double* maxerr,
                        int* nrunning) {
  if (!ctx || !B) return fail(ctx, ATLASGPU_EINVAL, "batch_poll: null");
  cudaSetDevice(ctx->device);
  std::vector<BatchCtl> c(B->nslots);
  CK(cudaMemcpyAsync(c.data(), B->d.ctl, c.size() * sizeof(BatchCtl), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  int run = 0;
  for (int b = 0; b < B->nslots; ++b) {
    if (status) status[b] = c[b].status;
    if (iters) iters[b] = c[b].iter;
    if (maxerr) maxerr[b] = c[b].maxerr;
    run += c[b].status == ATLASGPU_SLOT_RUNNING;
  }
  if (nrunning) *nrunning = run;
  return 0;
}

int atlasgpu_batch_run(atlasgpu_ctx* ctx, atlasgpu_batch* B, int poll_every, int* status, int* iters,
                       double* maxerr) {
  if (!ctx || !B || poll_every < 1) return fail(ctx, ATLASGPU_EINVAL, "batch_run: bad argument");
  int r, run = 1;
  // every running slot stops by its cap, so kHist launches always suffice
  for (int done = 0; run > 0 && done <= kHist; done += poll_every) {
    if ((r = atlasgpu_batch_step(ctx, B, poll_every))) return r;
    if ((r = atlasgpu_batch_poll(ctx, B, status, iters, maxerr, &run))) return r;
  }
  return run > 0 ? fail(ctx, ATLASGPU_ESTATE, "batch_run: %d slots still running", run) : 0;
}

int atlasgpu_batch_get(atlasgpu_ctx* ctx, atlasgpu_batch* B, int slot, double* t, double* rhox, double* p,
                       double* xne, double* flxerr, double* hsurf, double* maxerr_hist) {
  if (!ctx || !B || slot < 0 || slot >= B->nslots) return fail(ctx, ATLASGPU_EINVAL, "batch_get: bad slot");
  cudaSetDevice(ctx->device);
  const int kw = B->kw;
  std::vector<double> h((size_t)kNState * kw);
  BatchCtl c;
  CK(cudaMemcpyAsync(h.data(), B->state + (size_t)slot * kNState * kw, h.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&c, B->d.ctl + slot, sizeof c, cudaMemcpyDeviceToHost, ctx->stream));
  if (hsurf)
    CK(cudaMemcpyAsync(hsurf, B->d.hsurf + (size_t)slot * B->numnu, B->numnu * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream));
  std::vector<double> hist(kHist);
  if (maxerr_hist)
    CK(cudaMemcpyAsync(hist.data(), B->d.hist + (size_t)slot * kHist, kHist * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (t) memcpy(t, h.data() + 0 * kw, B->nrhox * sizeof(double));
  if (rhox) memcpy(rhox, h.data() + 1 * kw, B->nrhox * sizeof(double));
  if (p) memcpy(p, h.data() + 2 * kw, B->nrhox * sizeof(double));
  if (xne) memcpy(xne, h.data() + 3 * kw, B->nrhox * sizeof(double));
  if (flxerr) memcpy(flxerr, h.data() + 12 * kw, B->nrhox * sizeof(double));
  if (maxerr_hist) memcpy(maxerr_hist, hist.data(), std::min(c.iter, kHist) * sizeof(double));
  return 0;
}

int atlasgpu_batch_nslots(atlasgpu_batch* B) { return B ? B->nslots : ATLASGPU_EINVAL; }

}  // extern "C"
