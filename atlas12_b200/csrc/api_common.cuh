// api_common.cuh -- the context object behind the C ABI and its helpers.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstring>
#include <initializer_list>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"

struct atlasgpu_ctx {
  int device = 0;
  int precision = ATLASGPU_PREC_MIXED;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  int64_t launches = 0;
  bool timing = false;
  std::map<std::string, double> kms;
  std::map<std::string, double> kwork;  // counted work units of timed launches
  // named device buffers, grow-only
  std::map<std::string, std::pair<void*, size_t>> bufs;
  atlasgpu::JoshOps* ops = nullptr;  // device
  bool ops_set = false;
  bool kapp_set = false;     // atlasgpu_atlas_set_kapp_tables done
  bool kapp_h2_set = false;  // atlasgpu_atlas_set_kapp_h2_tables done
  bool atlas_stehle = false;  // atlasgpu_atlas_set_stehle_tables loaded tables
  int nsm = 148;
  size_t smem_optin = 0;
  // SELECTLINES tables (atlasgpu_atlas_select_tables)
  bool sel_ready = false;
  int sel_nwave = 0, sel_nspec = 0;
  double sel_hckt_last = 0.0;
  std::vector<double> sel_freqtab;   // CLIGHT_NMS / WAVETAB(k)
  std::vector<int16_t> sel_igrtab;   // H2O's IGR after advancing past bin k
};

namespace atlasgpu {

inline int fail(atlasgpu_ctx* c, int code, const char* fmt, ...) {
  char b[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(b, sizeof b, fmt, ap);
  va_end(ap);
  if (c) c->err = b;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return ::atlasgpu::fail(ctx, ATLASGPU_ECUDA, "%s: %s (%s:%d)", #call,              \
                              cudaGetErrorString(e_), __FILE__, __LINE__);                \
  } while (0)

#define CKL(ctx_)                                                                         \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess)                                                                \
      return ::atlasgpu::fail(ctx_, ATLASGPU_ECUDA, "launch: %s (%s:%d)",                \
                              cudaGetErrorString(e_), __FILE__, __LINE__);                \
    (ctx_)->launches++;                                                                   \
  } while (0)

// grow-only named device buffer
inline int buf(atlasgpu_ctx* ctx, const char* name, size_t bytes, void** out) {
  auto it = ctx->bufs.find(name);
  if (it != ctx->bufs.end() && it->second.second >= bytes) {
    *out = it->second.first;
    return 0;
  }
  if (it != ctx->bufs.end()) {
    cudaFree(it->second.first);
    ctx->bufs.erase(it);
  }
  void* p = nullptr;
  size_t want = bytes < 256 ? 256 : bytes;
  if (cudaMalloc(&p, want) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, ATLASGPU_ENOMEM, "cudaMalloc(%zu) failed for %s", want, name);
  }
  ctx->bufs[name] = {p, want};
  *out = p;
  return 0;
}

template <class T>
inline int bufT(atlasgpu_ctx* ctx, const char* name, size_t count, T** out) {
  void* p;
  int r = buf(ctx, name, count * sizeof(T), &p);
  *out = (T*)p;
  return r;
}

// CUDA-event timing of one named launch family (only when enabled)
// (accumulate = true adds to the family's time instead of replacing it: the
// caller clears the entry once per call for launches made in several parts)
struct Timer {
  atlasgpu_ctx* ctx;
  const char* name;
  bool acc;
  cudaEvent_t a = nullptr, b = nullptr;
  Timer(atlasgpu_ctx* c, const char* n, bool accumulate = false) : ctx(c), name(n), acc(accumulate) {
    if (ctx->timing) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, ctx->stream);
    }
  }
  void stop() {
    if (ctx->timing && a) {
      cudaEventRecord(b, ctx->stream);
      cudaEventSynchronize(b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (acc) ctx->kms[name] += ms;
      else ctx->kms[name] = ms;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      a = b = nullptr;
    }
  }
  ~Timer() { stop(); }
};

// Work counters of a timed launch family: a zeroed device array of n
// counters while timing is enabled, null otherwise (kernels then count
// nothing).  work_collect copies them back into ctx->kwork under the names.
inline unsigned long long* work_counters(atlasgpu_ctx* ctx, int n) {
  if (!ctx->timing) return nullptr;
  unsigned long long* p;
  if (bufT(ctx, "work_cnt", (size_t)n, &p)) return nullptr;
  if (cudaMemsetAsync(p, 0, n * sizeof(unsigned long long), ctx->stream) != cudaSuccess) return nullptr;
  return p;
}
inline void work_collect(atlasgpu_ctx* ctx, const unsigned long long* d, std::initializer_list<const char*> names) {
  if (!d) return;
  unsigned long long h[8] = {0};
  const int n = (int)names.size() < 8 ? (int)names.size() : 8;
  if (cudaMemcpyAsync(h, d, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return;
  int k = 0;
  for (const char* nm : names) {
    if (k >= n) break;
    ctx->kwork[nm] = (double)h[k++];
  }
}

inline int grid_for(atlasgpu_ctx* ctx, int64_t work, int threads, int per_sm = 8) {
  int64_t g = (work + threads - 1) / threads;
  int64_t cap = (int64_t)ctx->nsm * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

inline bool finite_all(const double* p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!(p[i] - p[i] == 0.0)) return false;
  return true;
}

// TABVOIGT's H0, H1, H2 packed as FP32 (H0, H1, H2, 0) for the mixed-precision LINOP1 walk
inline std::vector<float4> pack_voigt_f32(const double* h0, const double* h1, const double* h2, int n) {
  std::vector<float4> v(n);
  for (int i = 0; i < n; ++i) v[i] = make_float4((float)h0[i], (float)h1[i], (float)h2[i], 0.0f);
  return v;
}

// TABLOG (atlas12_modules.f90:2083-2086) for every INTEGER(2), index I + 32768, on the context
int ensure_tablog(atlasgpu_ctx* ctx, double** out);

// the four Stehle series to the device (api_synthe.cu): buffers named after
// prefix, *out the StehleDev[4] array; who names the caller in errors
int stehle_upload(atlasgpu_ctx* ctx, const atlasgpu_stehle_series* stehle, const char* prefix, const char* who,
                  StehleDev** out);

struct AtlasLine;
int atlas_prep_lines(atlasgpu_ctx* ctx, const int32_t* d_ld, const int32_t* h_ld, int64_t n,
                     const double* d_tablog, const double* d_ws, const double* h_ws, int numnu,
                     const int32_t* d_iwt, int nwave, int nspec, AtlasLine* d_lines);

}  // namespace atlasgpu
