// mlp.cu -- the learned warm start's network: a dense tanh MLP
// (nin -> nh1 -> nh2 -> nout, FP32 weights) with hand-written forward,
// backward and Adam kernels.  It maps stellar parameters to a starting
// structure; the unmodified ATLAS12 iteration still judges convergence, so
// the network only shortens the iteration.  No reference counterpart (the
// reference starts from a tabulated model).
//
// Layers: h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), y = W3 h2 + b3,
// W_l stored [out][in] row-major.  Loss: mean over samples and outputs of
// (y - target)^2.  Every sum runs in a fixed order (tile by tile, then a
// fixed-order reduction of per-block partials), so results repeat exactly.
#include <cmath>
#include <vector>

#include "api_common.cuh"

using namespace atlasgpu;

struct atlasgpu_mlp {
  int nin, nh1, nh2, nout;
  int64_t nparam;
  float *w, *g, *m, *v;   // parameters, gradient, Adam moments [nparam]
  int64_t step = 0;
  // activations / gradients for up to cap samples
  int cap = 0;
  float *x, *t, *h1, *h2, *y, *d1, *d2, *dy, *lpart;
};

namespace {

constexpr int kT = 32;  // tile edge

// C[m][n] (+)= sum_k A(m,k) B(k,n) with A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn]; epilogue: + bias[n], then tanh when act.
// mode 0: C = result; 1: C = result * (1 - Pact(m,n)^2) (tanh derivative
// of the layer output Pact, row-major [m][n]).
__global__ void k_gemm(int M, int N, int K, const float* __restrict__ A, int sam, int sak,
                       const float* __restrict__ B, int sbk, int sbn, const float* __restrict__ bias, int act,
                       int mode, const float* __restrict__ pact, float* __restrict__ C) {
  __shared__ float As[kT][kT + 1], Bs[kT][kT + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  const int m0 = blockIdx.y * kT, n0 = blockIdx.x * kT;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += kT) {
    for (int r = ty; r < kT; r += 8) {
      const int mm = m0 + r, kk = k0 + tx;
      As[r][tx] = (mm < M && kk < K) ? A[(size_t)mm * sam + (size_t)kk * sak] : 0.f;
      const int kb = k0 + r, nn = n0 + tx;
      Bs[r][tx] = (kb < K && nn < N) ? B[(size_t)kb * sbk + (size_t)nn * sbn] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ty + 8 * q;
      float s = acc[q];
#pragma unroll 8
      for (int kk = 0; kk < kT; ++kk) s = fmaf(As[r][kk], Bs[kk][tx], s);
      acc[q] = s;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int mm = m0 + ty + 8 * q, nn = n0 + tx;
    if (mm < M && nn < N) {
      float v = acc[q];
      if (bias) v += bias[nn];
      if (act) v = tanhf(v);
      if (mode == 1) {
        const float p = pact[(size_t)mm * N + nn];
        v = v * (1.f - p * p);
      }
      C[(size_t)mm * N + nn] = v;
    }
  }
}

// column sums: out[n] = sum_m A[m][n] (bias gradients), fixed order in m
__global__ void k_colsum(int M, int N, const float* __restrict__ A, float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; ++m) s += A[(size_t)m * N + n];
  out[n] = s;
}

// dy = 2 (y - t) / (n * nout); per-block partial sums of (y - t)^2
__global__ void k_mse(int64_t total, float scale, const float* __restrict__ y, const float* __restrict__ t,
                      float* __restrict__ dy, float* __restrict__ part) {
  __shared__ float sh[256];
  float s = 0.f;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const float d = y[e] - t[e];
    if (dy) dy[e] = 2.f * d * scale;
    s += d * d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sum_parts(int n, const float* __restrict__ part, float scale, float* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < n; ++i) s += part[i];
    *out = s * scale;
  }
}

__global__ void k_adam(int64_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// gather rows idx[0..n) of src [*][w] into dst [n][w]
__global__ void k_gather(int n, int w, const int* __restrict__ idx, const float* __restrict__ src,
                         float* __restrict__ dst) {
  const int64_t total = (int64_t)n * w;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / w), c = (int)(e % w);
    dst[e] = src[(size_t)idx[r] * w + c];
  }
}

struct Off {
  int64_t w1, b1, w2, b2, w3, b3;
};
Off offsets(const atlasgpu_mlp* p) {
  Off o;
  o.w1 = 0;
  o.b1 = o.w1 + (int64_t)p->nh1 * p->nin;
  o.w2 = o.b1 + p->nh1;
  o.b2 = o.w2 + (int64_t)p->nh2 * p->nh1;
  o.w3 = o.b2 + p->nh2;
  o.b3 = o.w3 + (int64_t)p->nout * p->nh2;
  return o;
}

int gemm(atlasgpu_ctx* ctx, int M, int N, int K, const float* A, int sam, int sak, const float* B, int sbk, int sbn,
         const float* bias, int act, int mode, const float* pact, float* C) {
  dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT), block(kT, 8);
  k_gemm<<<grid, block, 0, ctx->stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, act, mode, pact, C);
  CKL(ctx);
  return 0;
}

int ensure_cap(atlasgpu_ctx* ctx, atlasgpu_mlp* p, int n) {
  if (n <= p->cap) return 0;
  float** bufs[] = {&p->x, &p->t, &p->h1, &p->h2, &p->y, &p->d1, &p->d2, &p->dy};
  for (float** b : bufs)
    if (*b) cudaFree(*b);
  const int widths[] = {p->nin, p->nout, p->nh1, p->nh2, p->nout, p->nh1, p->nh2, p->nout};
  for (int i = 0; i < 8; ++i)
    if (cudaMalloc(bufs[i], sizeof(float) * (size_t)n * widths[i]) != cudaSuccess)
      return fail(ctx, ATLASGPU_ENOMEM, "mlp: activations for %d samples", n);
  p->cap = n;
  return 0;
}

// forward over n samples already in p->x
int forward(atlasgpu_ctx* ctx, atlasgpu_mlp* p, int n) {
  const Off o = offsets(p);
  int r;
  if ((r = gemm(ctx, n, p->nh1, p->nin, p->x, p->nin, 1, p->w + o.w1, 1, p->nin, p->w + o.b1, 1, 0, nullptr, p->h1)))
    return r;
  if ((r = gemm(ctx, n, p->nh2, p->nh1, p->h1, p->nh1, 1, p->w + o.w2, 1, p->nh1, p->w + o.b2, 1, 0, nullptr, p->h2)))
    return r;
  return gemm(ctx, n, p->nout, p->nh2, p->h2, p->nh2, 1, p->w + o.w3, 1, p->nh2, p->w + o.b3, 0, 0, nullptr, p->y);
}

// loss and gradient (p->g) over n samples in p->x, p->t; loss to *d_loss (device)
int backward(atlasgpu_ctx* ctx, atlasgpu_mlp* p, int n, float* d_loss) {
  const Off o = offsets(p);
  int r;
  const int64_t total = (int64_t)n * p->nout;
  const int nb = 64;
  k_mse<<<nb, 256, 0, ctx->stream>>>(total, 1.f / (float)total, p->y, p->t, p->dy, p->lpart);
  CKL(ctx);
  k_sum_parts<<<1, 32, 0, ctx->stream>>>(nb, p->lpart, 1.f / (float)total, d_loss);
  CKL(ctx);
  // layer 3: dW3 = dy^T h2, db3 = colsum dy, d2 = (dy W3) * (1 - h2^2)
  if ((r = gemm(ctx, p->nout, p->nh2, n, p->dy, 1, p->nout, p->h2, p->nh2, 1, nullptr, 0, 0, nullptr, p->g + o.w3)))
    return r;
  k_colsum<<<(p->nout + 127) / 128, 128, 0, ctx->stream>>>(n, p->nout, p->dy, p->g + o.b3);
  CKL(ctx);
  if ((r = gemm(ctx, n, p->nh2, p->nout, p->dy, p->nout, 1, p->w + o.w3, p->nh2, 1, nullptr, 0, 1, p->h2, p->d2)))
    return r;
  // layer 2
  if ((r = gemm(ctx, p->nh2, p->nh1, n, p->d2, 1, p->nh2, p->h1, p->nh1, 1, nullptr, 0, 0, nullptr, p->g + o.w2)))
    return r;
  k_colsum<<<(p->nh2 + 127) / 128, 128, 0, ctx->stream>>>(n, p->nh2, p->d2, p->g + o.b2);
  CKL(ctx);
  if ((r = gemm(ctx, n, p->nh1, p->nh2, p->d2, p->nh2, 1, p->w + o.w2, p->nh1, 1, nullptr, 0, 1, p->h1, p->d1)))
    return r;
  // layer 1
  if ((r = gemm(ctx, p->nh1, p->nin, n, p->d1, 1, p->nh1, p->x, p->nin, 1, nullptr, 0, 0, nullptr, p->g + o.w1)))
    return r;
  k_colsum<<<(p->nh1 + 127) / 128, 128, 0, ctx->stream>>>(n, p->nh1, p->d1, p->g + o.b1);
  CKL(ctx);
  return 0;
}

// splitmix64 for the initial weights (deterministic per seed)
uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

int atlasgpu_mlp_create(atlasgpu_ctx* ctx, int nin, int nh1, int nh2, int nout, uint64_t seed,
                        atlasgpu_mlp** out) {
  if (!ctx || !out || nin < 1 || nh1 < 1 || nh2 < 1 || nout < 1)
    return fail(ctx, ATLASGPU_EINVAL, "mlp_create: bad shape");
  *out = nullptr;
  cudaSetDevice(ctx->device);
  auto* p = new atlasgpu_mlp();
  p->nin = nin;
  p->nh1 = nh1;
  p->nh2 = nh2;
  p->nout = nout;
  const Off o = offsets(p);
  p->nparam = o.b3 + nout;
  float** bufs[] = {&p->w, &p->g, &p->m, &p->v};
  for (float** b : bufs)
    if (cudaMalloc(b, sizeof(float) * p->nparam) != cudaSuccess) {
      delete p;
      return fail(ctx, ATLASGPU_ENOMEM, "mlp_create");
    }
  CK(cudaMalloc(&p->lpart, sizeof(float) * 65));  // 64 block partials + the loss
  // Glorot-uniform weights, zero biases
  std::vector<float> h(p->nparam, 0.f);
  uint64_t s = seed;
  auto fill = [&](int64_t off, int fan_out, int fan_in) {
    const double lim = std::sqrt(6.0 / (fan_in + fan_out));
    for (int64_t i = 0; i < (int64_t)fan_out * fan_in; ++i) {
      const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
      h[off + i] = (float)((2.0 * u - 1.0) * lim);
    }
  };
  fill(o.w1, nh1, nin);
  fill(o.w2, nh2, nh1);
  fill(o.w3, nout, nh2);
  CK(cudaMemcpy(p->w, h.data(), sizeof(float) * p->nparam, cudaMemcpyHostToDevice));
  CK(cudaMemset(p->m, 0, sizeof(float) * p->nparam));
  CK(cudaMemset(p->v, 0, sizeof(float) * p->nparam));
  *out = p;
  return 0;
}

int atlasgpu_mlp_destroy(atlasgpu_ctx* ctx, atlasgpu_mlp* p) {
  if (!p) return ATLASGPU_EINVAL;
  if (ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
  }
  float* bufs[] = {p->w, p->g, p->m, p->v, p->x, p->t, p->h1, p->h2, p->y, p->d1, p->d2, p->dy, p->lpart};
  for (float* b : bufs)
    if (b) cudaFree(b);
  delete p;
  return 0;
}

int64_t atlasgpu_mlp_nparam(atlasgpu_mlp* p) { return p ? p->nparam : -1; }

int atlasgpu_mlp_get_params(atlasgpu_ctx* ctx, atlasgpu_mlp* p, float* out) {
  if (!ctx || !p || !out) return fail(ctx, ATLASGPU_EINVAL, "mlp_get_params");
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(out, p->w, sizeof(float) * p->nparam, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int atlasgpu_mlp_set_params(atlasgpu_ctx* ctx, atlasgpu_mlp* p, const float* in) {
  if (!ctx || !p || !in) return fail(ctx, ATLASGPU_EINVAL, "mlp_set_params");
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(p->w, in, sizeof(float) * p->nparam, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(p->m, 0, sizeof(float) * p->nparam, ctx->stream));
  CK(cudaMemsetAsync(p->v, 0, sizeof(float) * p->nparam, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  p->step = 0;
  return 0;
}

int atlasgpu_mlp_forward(atlasgpu_ctx* ctx, atlasgpu_mlp* p, const float* x, int n, float* y) {
  if (!ctx || !p || !x || !y || n < 1) return fail(ctx, ATLASGPU_EINVAL, "mlp_forward");
  cudaSetDevice(ctx->device);
  int r;
  if ((r = ensure_cap(ctx, p, n))) return r;
  CK(cudaMemcpyAsync(p->x, x, sizeof(float) * (size_t)n * p->nin, cudaMemcpyHostToDevice, ctx->stream));
  if ((r = forward(ctx, p, n))) return r;
  CK(cudaMemcpyAsync(y, p->y, sizeof(float) * (size_t)n * p->nout, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int atlasgpu_mlp_loss_grad(atlasgpu_ctx* ctx, atlasgpu_mlp* p, const float* x, const float* t, int n,
                           float* grad, float* loss) {
  if (!ctx || !p || !x || !t || n < 1) return fail(ctx, ATLASGPU_EINVAL, "mlp_loss_grad");
  cudaSetDevice(ctx->device);
  int r;
  if ((r = ensure_cap(ctx, p, n))) return r;
  CK(cudaMemcpyAsync(p->x, x, sizeof(float) * (size_t)n * p->nin, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(p->t, t, sizeof(float) * (size_t)n * p->nout, cudaMemcpyHostToDevice, ctx->stream));
  if ((r = forward(ctx, p, n))) return r;
  if ((r = backward(ctx, p, n, p->lpart + 64))) return r;
  if (grad) CK(cudaMemcpyAsync(grad, p->g, sizeof(float) * p->nparam, cudaMemcpyDeviceToHost, ctx->stream));
  float l = 0.f;
  CK(cudaMemcpyAsync(&l, p->lpart + 64, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (loss) *loss = l;
  return 0;
}

int atlasgpu_mlp_train(atlasgpu_ctx* ctx, atlasgpu_mlp* p, const float* x, const float* t, int n, int epochs,
                       int batch, float lr, uint64_t seed, float* loss_hist) {
  if (!ctx || !p || !x || !t || n < 1 || epochs < 0 || batch < 1)
    return fail(ctx, ATLASGPU_EINVAL, "mlp_train: bad argument");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  if (batch > n) batch = n;
  int r;
  if ((r = ensure_cap(ctx, p, batch))) return r;
  float *dx, *dt, *dloss;
  int* didx;
  CK(cudaMalloc(&dx, sizeof(float) * (size_t)n * p->nin));
  CK(cudaMalloc(&dt, sizeof(float) * (size_t)n * p->nout));
  CK(cudaMalloc(&didx, sizeof(int) * (size_t)n));
  CK(cudaMalloc(&dloss, sizeof(float) * (size_t)(epochs + 1)));
  CK(cudaMemcpyAsync(dx, x, sizeof(float) * (size_t)n * p->nin, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dt, t, sizeof(float) * (size_t)n * p->nout, cudaMemcpyHostToDevice, st));
  std::vector<int> perm(n);
  uint64_t s = seed;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs && r == 0; ++ep) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = n - 1; i > 0; --i) {  // Fisher-Yates with splitmix
      const int j = (int)(splitmix(s) % (uint64_t)(i + 1));
      std::swap(perm[i], perm[j]);
    }
    CK(cudaMemcpyAsync(didx, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));  // perm is rewritten next epoch
    for (int b0 = 0; b0 + batch <= n; b0 += batch) {
      k_gather<<<grid_for(ctx, (int64_t)batch * p->nin, 256, 4), 256, 0, st>>>(batch, p->nin, didx + b0, dx, p->x);
      k_gather<<<grid_for(ctx, (int64_t)batch * p->nout, 256, 4), 256, 0, st>>>(batch, p->nout, didx + b0, dt, p->t);
      CKL(ctx);
      if ((r = forward(ctx, p, batch)) || (r = backward(ctx, p, batch, dloss + ep))) break;
      p->step += 1;
      const float c1 = 1.f - powf(b1, (float)p->step), c2 = 1.f - powf(b2, (float)p->step);
      k_adam<<<grid_for(ctx, p->nparam, 256, 4), 256, 0, st>>>(p->nparam, p->w, p->g, p->m, p->v, lr, b1, b2, eps,
                                                               c1, c2);
      CKL(ctx);
    }
  }
  if (r == 0 && loss_hist && epochs > 0)
    CK(cudaMemcpyAsync(loss_hist, dloss, sizeof(float) * epochs, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  cudaFree(dx);
  cudaFree(dt);
  cudaFree(didx);
  cudaFree(dloss);
  return r;
}

}  // extern "C"
