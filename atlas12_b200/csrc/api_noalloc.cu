// api_noalloc.cu -- the frequency loop of the ATLAS12 RT pass for callers
// that cannot allocate device memory.
//
// Some callers manage every byte of device memory themselves and may not call
// cudaMalloc: a Fortran driver that owns its device arrays through its own
// allocator or memory pool, code running inside a memory budget enforced by
// the host application, or a process that must not grow its footprint after
// start-up.  atlasgpu_atlas_rt_pass_noalloc serves them: the caller passes all
// inputs and outputs as device pointers, and the only scratch the pass needs
// (one row of partial sums per thread group) lives in a fixed file-scope
// device array.
//
// That array is part of the library image: every GPU that loads the library
// holds it (kNoAllocRows x (8*kKwMax + 1) doubles = 6.6 MB) until the
// process exits.  All calls share it and it keeps the last call's contents;
// every row a call reads is written whole by that call first (the depths
// between nrhox and kw as zeros), so nothing needs clearing, but two calls
// that overlap on the GPU (different streams, or different host threads on
// one device) race on it and must be serialised by the caller.  The
// per-device address lookup itself is safe from several host threads.
#include <atomic>

#include "api_common.cuh"
#include "atlas.cuh"

using namespace atlasgpu;

namespace {

constexpr int kNoAllocRows = 1024;                // maximum thread groups (rows of partials)
constexpr int kNoAllocRow = kAcc * kKwMax + 1;    // one row: 8 sums per depth + PRADK0

static __device__ __align__(256) double g_noalloc_partial[(size_t)kNoAllocRows * kNoAllocRow];

constexpr int kMaxDevices = 64;
// device address of the array, per device; host threads making their first
// call at once may both look it up, and both store the same address
std::atomic<double*> g_partial_addr[kMaxDevices];

}  // namespace

extern "C" {

int atlasgpu_atlas_rt_pass_noalloc(atlasgpu_ctx* ctx, int numnu, const double* d_waveset,
                                   const double* d_rcoset, const double* d_acont, const double* d_sigmac,
                                   const double* d_scont, int kw, const double* d_xlines_t, int nrhox,
                                   const double* d_rhox, const double* d_t, const double* d_hkt, double teff,
                                   double* d_sums, double* d_hsurf) {
  if (!ctx) return ATLASGPU_EINVAL;
  if (!ctx->ops_set) return fail(ctx, ATLASGPU_ESTATE, "rt_pass_noalloc: operators not set");
  if (numnu < 1 || nrhox < 4 || kw < nrhox)
    return fail(ctx, ATLASGPU_EINVAL, "rt_pass_noalloc: numnu %d, nrhox %d, kw %d", numnu, nrhox, kw);
  if (kw > kKwMax)
    return fail(ctx, ATLASGPU_EINVAL, "rt_pass_noalloc: kw = %d exceeds the fixed scratch limit of %d depths",
                kw, kKwMax);
  if (!d_waveset || !d_rcoset || !d_acont || !d_sigmac || !d_xlines_t || !d_rhox || !d_t || !d_hkt || !d_sums ||
      !d_hsurf)
    return fail(ctx, ATLASGPU_EINVAL, "rt_pass_noalloc: null device pointer");
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return fail(ctx, ATLASGPU_EINVAL, "rt_pass_noalloc: device %d beyond %d", ctx->device, kMaxDevices);
  CK(cudaSetDevice(ctx->device));
  // set-up, once per device, with that device current: the host-side name of
  // the array is not a device address, so ask the runtime for the address
  double* partial = g_partial_addr[ctx->device].load(std::memory_order_acquire);
  if (!partial) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partial);
    if (e != cudaSuccess || !p)
      return fail(ctx, ATLASGPU_ECUDA, "rt_pass_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    partial = (double*)p;
    g_partial_addr[ctx->device].store(partial, std::memory_order_release);
  }
  // launch shape: at most kNoAllocRows thread groups (rows of partials),
  // contiguous frequencies per group
  const size_t smem = rt_smem_bytes();
  int target = ctx->nsm * kRtMinBlocks * kRtGroups * 4;
  if (target > kNoAllocRows) target = kNoAllocRows;
  const int npw = (numnu + target - 1) / target;
  const int ng = (numnu + npw - 1) / npw;
  const int blocks = (ng + kRtGroups - 1) / kRtGroups;
  const int nwl = blocks * kRtGroups;
  if (nwl > kNoAllocRows)
    return fail(ctx, ATLASGPU_EINVAL, "rt_pass_noalloc: %d thread groups exceed the scratch limit %d", nwl,
                kNoAllocRows);
  CK(cudaFuncSetAttribute(k_atlas_rt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  RtArgs a{ctx->ops, numnu, nrhox, kw, d_waveset, d_rcoset, d_acont, d_sigmac, d_scont, d_xlines_t,
           d_rhox, d_t, d_hkt, teff, npw, numnu, 1, partial, d_hsurf, nullptr};
  k_atlas_rt<<<blocks, kRtThreads, smem, ctx->stream>>>(a);
  CKL(ctx);
  launch_reduce(partial, nwl, kw, d_sums, ctx->stream);
  CKL(ctx);
  return ATLASGPU_OK;
}

}  // extern "C"
