// The learned window planner: a three-layer perceptron
//
//   h1 = relu(W1 x + b1),  h2 = relu(W2 h1 + b2),  y = W3 h2 + b3
//
// with BF16 weights and FP32 arithmetic (every product of a BF16 weight and an FP32
// activation accumulates in FP32), trained on the GPU by these kernels: forward, the two
// backward products, the weighted squared-error loss and Adam on FP32 master weights
// whose BF16 copies the forward and backward passes read.  An extension: the reference
// chooses filter degree and subspace size by hand.
//
// Every product is one tiled FP32 GEMM kernel, C = op(A) op(B) (+ bias, relu or a relu
// mask), with 64 x 64 output tiles, 16-deep K slices staged in shared memory and a 4 x 4
// register micro-tile per thread.  The network is small (about 0.2 M parameters) and
// the batches a few thousand rows, so these products are latency- rather than
// throughput-bound and FP32 FMA on the CUDA cores is the right unit.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>

#include "sma_internal.h"

namespace sma {

namespace {

constexpr int kTile = 64, kDepth = 16;

__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }

// C[m, n] (ldc) = sum_k A(m, k) B(k, n), A(m, k) = transA ? A[k*lda + m] : A[m*lda + k],
// B(k, n) = transB ? B[n*ldb + k] : B[k*ldb + n]; epilogue: + bias[n], relu, or times
// (mask[m*ldm + n] > 0).
template <typename TB, bool TA_, bool TB_>
__global__ void __launch_bounds__(256)
gemm_kernel(int64_t M, int64_t N, int64_t K, const float *__restrict__ A, int64_t lda,
            const TB *__restrict__ B, int64_t ldb, float *__restrict__ C, int64_t ldc,
            const float *__restrict__ bias, int relu, const float *__restrict__ mask,
            int64_t ldm) {
  __shared__ float As[kDepth][kTile + 1];
  __shared__ float Bs[kDepth][kTile + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int64_t m0 = (int64_t)blockIdx.y * kTile, n0 = (int64_t)blockIdx.x * kTile;
  float acc[4][4] = {};
  for (int64_t k0 = 0; k0 < K; k0 += kDepth) {
    for (int e = threadIdx.x; e < kDepth * kTile; e += 256) {
      const int kk = e / kTile, mm = e % kTile;
      const int64_t gm = m0 + mm, gk = k0 + kk;
      float a = 0.f;
      if (gm < M && gk < K) a = TA_ ? A[gk * lda + gm] : A[gm * lda + gk];
      As[kk][mm] = a;
      const int64_t gn = n0 + mm;
      float b = 0.f;
      if (gn < N && gk < K) b = to_f(TB_ ? B[gn * ldb + gk] : B[gk * ldb + gn]);
      Bs[kk][mm] = b;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kDepth; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t gn = n0 + tx + 16 * j;
      if (gn >= N) continue;
      float v = acc[i][j];
      if (bias) v += bias[gn];
      if (relu) v = fmaxf(v, 0.f);
      if (mask && !(mask[gm * ldm + gn] > 0.f)) v = 0.f;
      C[gm * ldc + gn] = v;
    }
  }
}

template <typename TB, bool TA_, bool TB_>
void gemm(cudaStream_t st, int64_t M, int64_t N, int64_t K, const float *A, int64_t lda,
          const TB *B, int64_t ldb, float *C, int64_t ldc, const float *bias, bool relu,
          const float *mask, int64_t ldm) {
  if (M == 0 || N == 0) return;
  dim3 grid((unsigned)((N + kTile - 1) / kTile), (unsigned)((M + kTile - 1) / kTile));
  gemm_kernel<TB, TA_, TB_><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias,
                                                   relu ? 1 : 0, mask, ldm);
  SMA_CHECK_LAUNCH();
}

// out[n] = sum_m X[m*ld + n] (bias gradients), one thread per column, fixed order.
__global__ void colsum_kernel(int64_t M, int64_t N, const float *__restrict__ X, int64_t ld,
                              float *__restrict__ out) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int64_t m = 0; m < M; ++m) s += X[m * ld + n];
  out[n] = s;
}

// dY = (2 / B) w (Y - T); partial[b] = sum_o w (Y - T)^2 for row b.
__global__ void mse_kernel(int64_t Bn, int64_t O, const float *__restrict__ Y,
                           const float *__restrict__ T, const float *__restrict__ w,
                           float *__restrict__ dY, float *__restrict__ partial) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= Bn) return;
  float s = 0.f;
  for (int64_t o = 0; o < O; ++o) {
    const float r = Y[b * O + o] - T[b * O + o];
    const float wt = w ? w[b * O + o] : 1.f;
    s += wt * r * r;
    dY[b * O + o] = 2.f * wt * r / (float)Bn;
  }
  partial[b] = s;
}

// loss[0] = (1/B) sum_b partial[b], one block, fixed order
__global__ void loss_reduce_kernel(int64_t Bn, const float *__restrict__ partial,
                                   float *__restrict__ loss) {
  __shared__ float sh[256];
  float s = 0.f;
  for (int64_t b = threadIdx.x; b < Bn; b += 256) s += partial[b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = sh[0] / (float)Bn;
}

__global__ void to_bf16_kernel(int64_t n, const float *__restrict__ x, __nv_bfloat16 *__restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

// Adam (Kingma & Ba 2015) with bias correction on FP32 masters; writes the BF16 copies.
__global__ void adam_kernel(int64_t n, float *__restrict__ p, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v,
                            __nv_bfloat16 *__restrict__ pb, float lr, float b1, float b2,
                            float eps, float c1, float c2, float wd) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + wd * p[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float q = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = q;
  pb[i] = __float2bfloat16_rn(q);
}

// rows of X (ld in_dim) picked by idx into Xs; the same for T and w (ld out_dim)
__global__ void gather_rows_kernel(int64_t Bn, int64_t D, const float *__restrict__ X,
                                   const int64_t *__restrict__ idx, float *__restrict__ Xs) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= Bn * D) return;
  const int64_t b = t / D, d = t % D;
  Xs[t] = X[idx[b] * D + d];
}

inline unsigned blocks(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

}  // namespace
}  // namespace sma

namespace sma {

void mlp_init(sma_mlp *net, int64_t in, int64_t hid, int64_t out, uint64_t seed) {
  net->in = in;
  net->hid = hid;
  net->out = out;
  net->oW1 = 0;
  net->ob1 = net->oW1 + hid * in;
  net->oW2 = net->ob1 + hid;
  net->ob2 = net->oW2 + hid * hid;
  net->oW3 = net->ob2 + hid;
  net->ob3 = net->oW3 + out * hid;
  net->nparam = net->ob3 + out;
  cudaStream_t st = net->ctx->stream;
  net->master.alloc(net->nparam, st);
  net->grad.alloc(net->nparam, st);
  net->m.alloc(net->nparam, st);
  net->v.alloc(net->nparam, st);
  net->wbf.alloc(net->nparam, st);
  // He-uniform hidden layers, a zero output layer (the untrained network predicts 0)
  std::vector<float> p(net->nparam, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int64_t off, int64_t rows, int64_t cols) {
    const double lim = std::sqrt(6.0 / (double)cols);
    std::uniform_real_distribution<double> u(-lim, lim);
    for (int64_t i = 0; i < rows * cols; ++i) p[off + i] = (float)u(rng);
  };
  fill(net->oW1, hid, in);
  fill(net->oW2, hid, hid);
  SMA_CUDA(cudaMemcpyAsync(net->master.p, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  SMA_CUDA(cudaMemsetAsync(net->m.p, 0, net->nparam * sizeof(float), st));
  SMA_CUDA(cudaMemsetAsync(net->v.p, 0, net->nparam * sizeof(float), st));
  to_bf16_kernel<<<blocks(net->nparam), 256, 0, st>>>(net->nparam, net->master.p, net->wbf.p);
  SMA_CHECK_LAUNCH();
  SMA_CUDA(cudaStreamSynchronize(st));
}

void mlp_set_params(sma_mlp *net, const float *p) {
  cudaStream_t st = net->ctx->stream;
  SMA_CUDA(cudaMemcpyAsync(net->master.p, p, net->nparam * sizeof(float), cudaMemcpyHostToDevice, st));
  to_bf16_kernel<<<blocks(net->nparam), 256, 0, st>>>(net->nparam, net->master.p, net->wbf.p);
  SMA_CHECK_LAUNCH();
  SMA_CUDA(cudaMemsetAsync(net->m.p, 0, net->nparam * sizeof(float), st));
  SMA_CUDA(cudaMemsetAsync(net->v.p, 0, net->nparam * sizeof(float), st));
  net->adam_t = 0;
  SMA_CUDA(cudaStreamSynchronize(st));
}

// forward on a device batch X (B x in); the output lands in net->y
static void mlp_forward_dev(sma_mlp *net, const float *X, int64_t B) {
  cudaStream_t st = net->ctx->stream;
  net->ensure(B);
  const __nv_bfloat16 *w = net->wbf.p;
  const float *bias = net->master.p;  // biases are used in FP32
  gemm<__nv_bfloat16, false, true>(st, B, net->hid, net->in, X, net->in, w + net->oW1, net->in,
                                   net->h1.p, net->hid, bias + net->ob1, true, nullptr, 0);
  gemm<__nv_bfloat16, false, true>(st, B, net->hid, net->hid, net->h1.p, net->hid, w + net->oW2,
                                   net->hid, net->h2.p, net->hid, bias + net->ob2, true, nullptr, 0);
  gemm<__nv_bfloat16, false, true>(st, B, net->out, net->hid, net->h2.p, net->hid, w + net->oW3,
                                   net->hid, net->y.p, net->out, bias + net->ob3, false, nullptr, 0);
}

// loss and gradient of the packed parameters for a device batch
static void mlp_backward_dev(sma_mlp *net, const float *X, const float *T, const float *wt,
                             int64_t B) {
  cudaStream_t st = net->ctx->stream;
  const __nv_bfloat16 *w = net->wbf.p;
  float *g = net->grad.p;
  mse_kernel<<<blocks(B), 256, 0, st>>>(B, net->out, net->y.p, T, wt, net->dy.p, net->partial.p);
  SMA_CHECK_LAUNCH();
  loss_reduce_kernel<<<1, 256, 0, st>>>(B, net->partial.p, net->loss.p);
  SMA_CHECK_LAUNCH();
  // layer 3: dW3 = dy^T h2, db3 = colsum dy, d2 = (dy W3) * [h2 > 0]
  gemm<float, true, false>(st, net->out, net->hid, B, net->dy.p, net->out, net->h2.p, net->hid,
                           g + net->oW3, net->hid, nullptr, false, nullptr, 0);
  colsum_kernel<<<blocks(net->out), 256, 0, st>>>(B, net->out, net->dy.p, net->out, g + net->ob3);
  SMA_CHECK_LAUNCH();
  gemm<__nv_bfloat16, false, false>(st, B, net->hid, net->out, net->dy.p, net->out, w + net->oW3,
                                    net->hid, net->d2.p, net->hid, nullptr, false, net->h2.p, net->hid);
  // layer 2
  gemm<float, true, false>(st, net->hid, net->hid, B, net->d2.p, net->hid, net->h1.p, net->hid,
                           g + net->oW2, net->hid, nullptr, false, nullptr, 0);
  colsum_kernel<<<blocks(net->hid), 256, 0, st>>>(B, net->hid, net->d2.p, net->hid, g + net->ob2);
  SMA_CHECK_LAUNCH();
  gemm<__nv_bfloat16, false, false>(st, B, net->hid, net->hid, net->d2.p, net->hid, w + net->oW2,
                                    net->hid, net->d1.p, net->hid, nullptr, false, net->h1.p, net->hid);
  // layer 1
  gemm<float, true, false>(st, net->hid, net->in, B, net->d1.p, net->hid, X, net->in,
                           g + net->oW1, net->in, nullptr, false, nullptr, 0);
  colsum_kernel<<<blocks(net->hid), 256, 0, st>>>(B, net->hid, net->d1.p, net->hid, g + net->ob1);
  SMA_CHECK_LAUNCH();
}

void mlp_forward(sma_mlp *net, const float *X_host, int64_t B, float *Y_host) {
  cudaStream_t st = net->ctx->stream;
  DevBuf<float> X(B * net->in, st);
  SMA_CUDA(cudaMemcpyAsync(X.p, X_host, B * net->in * sizeof(float), cudaMemcpyHostToDevice, st));
  mlp_forward_dev(net, X.p, B);
  SMA_CUDA(cudaMemcpyAsync(Y_host, net->y.p, B * net->out * sizeof(float), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
}

float mlp_grad(sma_mlp *net, const float *X_host, const float *T_host, const float *w_host,
               int64_t B, float *grad_host) {
  cudaStream_t st = net->ctx->stream;
  DevBuf<float> X(B * net->in, st), T(B * net->out, st), W(w_host ? B * net->out : 0, st);
  SMA_CUDA(cudaMemcpyAsync(X.p, X_host, B * net->in * sizeof(float), cudaMemcpyHostToDevice, st));
  SMA_CUDA(cudaMemcpyAsync(T.p, T_host, B * net->out * sizeof(float), cudaMemcpyHostToDevice, st));
  if (w_host)
    SMA_CUDA(cudaMemcpyAsync(W.p, w_host, B * net->out * sizeof(float), cudaMemcpyHostToDevice, st));
  mlp_forward_dev(net, X.p, B);
  mlp_backward_dev(net, X.p, T.p, w_host ? W.p : nullptr, B);
  float loss = 0.f;
  SMA_CUDA(cudaMemcpyAsync(&loss, net->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
  if (grad_host)
    SMA_CUDA(cudaMemcpyAsync(grad_host, net->grad.p, net->nparam * sizeof(float), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  return loss;
}

// Minibatch Adam on the GPU over a host data set of N rows; loss_hist[s] is the minibatch
// loss before step s.  Minibatches are drawn without replacement from a seeded
// permutation per epoch.
void mlp_train(sma_mlp *net, const float *X_host, const float *T_host, const float *w_host,
               int64_t N, int64_t steps, double lr, int64_t mb, uint64_t seed, double weight_decay,
               float *loss_hist) {
  cudaStream_t st = net->ctx->stream;
  require(N >= 1 && mb >= 1 && steps >= 0, SMA_ERR_ARG, "bad training sizes");
  mb = std::min(mb, N);
  DevBuf<float> X(N * net->in, st), T(N * net->out, st), W(w_host ? N * net->out : 0, st);
  DevBuf<float> Xs(mb * net->in, st), Ts(mb * net->out, st), Ws(w_host ? mb * net->out : 0, st);
  DevBuf<float> hist(std::max<int64_t>(steps, 1), st);
  SMA_CUDA(cudaMemcpyAsync(X.p, X_host, N * net->in * sizeof(float), cudaMemcpyHostToDevice, st));
  SMA_CUDA(cudaMemcpyAsync(T.p, T_host, N * net->out * sizeof(float), cudaMemcpyHostToDevice, st));
  if (w_host)
    SMA_CUDA(cudaMemcpyAsync(W.p, w_host, N * net->out * sizeof(float), cudaMemcpyHostToDevice, st));
  // all minibatch index lists of the run, drawn up front
  const int64_t per_epoch = N / mb;
  std::vector<int64_t> idx((size_t)steps * mb);
  std::mt19937_64 rng(seed);
  std::vector<int64_t> perm(N);
  for (int64_t s = 0; s < steps; ++s) {
    const int64_t e = per_epoch > 0 ? s % per_epoch : 0;
    if (e == 0) {
      std::iota(perm.begin(), perm.end(), 0);
      std::shuffle(perm.begin(), perm.end(), rng);
    }
    for (int64_t b = 0; b < mb; ++b) idx[s * mb + b] = perm[e * mb + b];
  }
  DevBuf<int64_t> didx(std::max<size_t>(idx.size(), 1), st);
  if (!idx.empty())
    SMA_CUDA(cudaMemcpyAsync(didx.p, idx.data(), idx.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  const float b1 = 0.9f, b2 = 0.999f;
  for (int64_t s = 0; s < steps; ++s) {
    const int64_t *ix = didx.p + s * mb;
    gather_rows_kernel<<<blocks(mb * net->in), 256, 0, st>>>(mb, net->in, X.p, ix, Xs.p);
    SMA_CHECK_LAUNCH();
    gather_rows_kernel<<<blocks(mb * net->out), 256, 0, st>>>(mb, net->out, T.p, ix, Ts.p);
    SMA_CHECK_LAUNCH();
    if (w_host) {
      gather_rows_kernel<<<blocks(mb * net->out), 256, 0, st>>>(mb, net->out, W.p, ix, Ws.p);
      SMA_CHECK_LAUNCH();
    }
    mlp_forward_dev(net, Xs.p, mb);
    mlp_backward_dev(net, Xs.p, Ts.p, w_host ? Ws.p : nullptr, mb);
    SMA_CUDA(cudaMemcpyAsync(hist.p + s, net->loss.p, sizeof(float), cudaMemcpyDeviceToDevice, st));
    net->adam_t += 1;
    const float c1 = 1.f - std::pow(b1, (float)net->adam_t), c2 = 1.f - std::pow(b2, (float)net->adam_t);
    adam_kernel<<<blocks(net->nparam), 256, 0, st>>>(net->nparam, net->master.p, net->grad.p,
                                                     net->m.p, net->v.p, net->wbf.p, (float)lr, b1,
                                                     b2, 1e-8f, c1, c2, (float)weight_decay);
    SMA_CHECK_LAUNCH();
  }
  if (loss_hist && steps > 0)
    SMA_CUDA(cudaMemcpyAsync(loss_hist, hist.p, steps * sizeof(float), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
}

void mlp_get_params(const sma_mlp *net, float *p) {
  cudaStream_t st = net->ctx->stream;
  SMA_CUDA(cudaMemcpyAsync(p, net->master.p, net->nparam * sizeof(float), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
}

}  // namespace sma
