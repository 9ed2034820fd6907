// mlp_train.cu -- training and loading of the learned con2prim seed.
//
// The network (mlp.cuh) is trained here by this library's own kernels:
// FP32 forward pass, backward pass (weight and bias gradients, tanh
// derivative), mean-squared loss on standardised targets and Adam.  The
// weight vector layout (ECHO_MLP_NWEIGHTS floats) is, layer by layer,
// W_l[K_l][N_l] row-major followed by b_l[N_l], with (K, N) = (6, 64),
// (64, 64) x3, (64, 2).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/echo_gpu.h"
#include "ctx.cuh"

#define CK(x)                                                                               \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) {                                                                \
      fprintf(stderr, "echo_gpu: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                    \
      return ECHO_ERR_CUDA;                                                                 \
    }                                                                                       \
  } while (0)

namespace {

constexpr int NL = 5, NIN = echo::MLP_NIN;
constexpr int LK[NL] = {NIN, 64, 64, 64, 64};
constexpr int LN[NL] = {64, 64, 64, 64, 2};
constexpr int WOFF[NL] = {0, 448, 4608, 8768, 12928};
constexpr int BOFF[NL] = {384, 4544, 8704, 12864, 13056};
static_assert(BOFF[NL - 1] + 2 == ECHO_MLP_NWEIGHTS, "weight vector layout");
static_assert(echo::MLP_PARAMS_N - echo::MLP_FMEAN == ECHO_MLP_NNORM, "norm layout");

// round-to-nearest-even float -> bf16 bits
unsigned short bf16_bits(float f) {
  unsigned u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (unsigned short)(u >> 16);
  unsigned r = u + 0x7fffu + ((u >> 16) & 1u);
  return (unsigned short)(r >> 16);
}

// B-operand fragments of mma.m16n8k16 (see mlp.cuh): for k-tile kt, n-tile
// nt and lane (g = lane/4, t = lane%4): .x = (W[k0][n], W[k0+1][n]),
// .y = (W[k0+8][n], W[k0+9][n]) with k0 = 16 kt + 2t, n = 8 nt + g; zero
// outside the layer's K x N.
void pack_layer(const float* W, int K, int N, int nkt, int nnt, unsigned* out) {
  auto w = [&](int k, int n) -> float { return (k < K && n < N) ? W[k * N + n] : 0.f; };
  for (int kt = 0; kt < nkt; kt++)
    for (int nt = 0; nt < nnt; nt++)
      for (int lane = 0; lane < 32; lane++) {
        int g = lane / 4, t = lane % 4, n = nt * 8 + g, k0 = kt * 16 + 2 * t;
        unsigned lo = bf16_bits(w(k0, n)) | ((unsigned)bf16_bits(w(k0 + 1, n)) << 16);
        unsigned hi = bf16_bits(w(k0 + 8, n)) | ((unsigned)bf16_bits(w(k0 + 9, n)) << 16);
        unsigned* o = out + ((size_t)(kt * nnt + nt) * 32 + lane) * 2;
        o[0] = lo;
        o[1] = hi;
      }
}

void pack_network(const float* W, const float* norm, std::vector<unsigned>& frag, std::vector<float>& par) {
  frag.assign(echo::MLP_FRAG_N, 0u);
  par.assign(echo::MLP_PARAMS_N, 0.f);
  pack_layer(W + WOFF[0], NIN, 64, 1, 8, frag.data() + echo::MLP_FRAG_L0);
  pack_layer(W + WOFF[1], 64, 64, 4, 8, frag.data() + echo::MLP_FRAG_L1);
  pack_layer(W + WOFF[2], 64, 64, 4, 8, frag.data() + echo::MLP_FRAG_L2);
  pack_layer(W + WOFF[3], 64, 64, 4, 8, frag.data() + echo::MLP_FRAG_L3);
  pack_layer(W + WOFF[4], 64, 2, 4, 1, frag.data() + echo::MLP_FRAG_L4);
  for (int l = 0; l < 4; l++)
    for (int n = 0; n < 64; n++) par[echo::MLP_B0 + l * 64 + n] = W[BOFF[l] + n];
  par[echo::MLP_B4 + 0] = W[BOFF[4] + 0];
  par[echo::MLP_B4 + 1] = W[BOFF[4] + 1];
  for (int j = 0; j < ECHO_MLP_NNORM; j++) par[echo::MLP_FMEAN + j] = norm[j];
}

// ---------------------------------------------------------------------------
// training kernels (FP32)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned hash32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

__global__ void k_gather(const float* Xs, const float* Ts, int n, int B, unsigned step, unsigned seed, float* A0,
                         float* Y) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  unsigned i = hash32(seed * 0x9e3779b9u ^ hash32(step * 1000003u + (unsigned)b)) % (unsigned)n;
  for (int j = 0; j < NIN; j++) A0[b * NIN + j] = Xs[(size_t)i * NIN + j];
  Y[b * 2 + 0] = Ts[(size_t)i * 2 + 0];
  Y[b * 2 + 1] = Ts[(size_t)i * 2 + 1];
}

// out[b][n] = act(bias[n] + sum_k A[b][k] W[k][n])
__global__ void k_linear(const float* A, const float* W, const float* bias, float* out, int B, int K, int N,
                         int act) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= B * N) return;
  int b = id / N, n = id % N;
  float z = bias[n];
  for (int k = 0; k < K; k++) z += A[b * K + k] * W[k * N + n];
  out[id] = act ? tanhf(z) : z;
}

// dO = d(loss)/dO for loss = mean (O - Y)^2 over B x 2 entries
__global__ void k_loss(const float* O, const float* Y, int B, float* dO, float* loss) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (id < B * 2) {
    float d = O[id] - Y[id];
    dO[id] = 2.f * d / (float)(B * 2);
    l = d * d / (float)(B * 2);
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// dW[k][n] = sum_b A[b][k] dZ[b][n]  (one block per (k, n))
__global__ void k_wgrad(const float* A, const float* dZ, int B, int K, int N, float* dW) {
  int k = blockIdx.x / N, n = blockIdx.x % N;
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) s += A[b * K + k] * dZ[b * N + n];
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    dW[k * N + n] = t;
  }
}

// db[n] = sum_b dZ[b][n]
__global__ void k_bgrad(const float* dZ, int B, int N, float* db) {
  int n = blockIdx.x;
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) s += dZ[b * N + n];
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    db[n] = t;
  }
}

// dZprev[b][k] = (sum_n dZ[b][n] W[k][n]) * (1 - Ain[b][k]^2)   (Ain = tanh output)
__global__ void k_backact(const float* dZ, const float* W, const float* Ain, int B, int K, int N, float* dZprev) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= B * K) return;
  int b = id / K, k = id % K;
  float s = 0.f;
  for (int n = 0; n < N; n++) s += dZ[b * N + n] * W[k * N + n];
  float a = Ain[id];
  dZprev[id] = s * (1.f - a * a);
}

__global__ void k_adam(float* W, const float* G, float* m, float* v, int n, float lr, float b1, float b2,
                       float eps, int t) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float g = G[i];
  m[i] = b1 * m[i] + (1.f - b1) * g;
  v[i] = b2 * v[i] + (1.f - b2) * g * g;
  float mh = m[i] / (1.f - powf(b1, (float)t));
  float vh = v[i] / (1.f - powf(b2, (float)t));
  W[i] -= lr * mh / (sqrtf(vh) + eps);
}

struct Trainer {
  int B = 0;
  float *W = nullptr, *G = nullptr, *m = nullptr, *v = nullptr;
  float* act[NL + 1] = {nullptr};  // act[0] = input (B x NIN), act[l+1] = layer l output
  float *dZ[NL] = {nullptr}, *Y = nullptr, *loss = nullptr;
  ~Trainer() {
    cudaFree(W);
    cudaFree(G);
    cudaFree(m);
    cudaFree(v);
    for (int l = 0; l <= NL; l++) cudaFree(act[l]);
    for (int l = 0; l < NL; l++) cudaFree(dZ[l]);
    cudaFree(Y);
    cudaFree(loss);
  }
  int alloc(int batch) {
    B = batch;
    CK(cudaMalloc(&W, sizeof(float) * ECHO_MLP_NWEIGHTS));
    CK(cudaMalloc(&G, sizeof(float) * ECHO_MLP_NWEIGHTS));
    CK(cudaMalloc(&m, sizeof(float) * ECHO_MLP_NWEIGHTS));
    CK(cudaMalloc(&v, sizeof(float) * ECHO_MLP_NWEIGHTS));
    CK(cudaMemset(m, 0, sizeof(float) * ECHO_MLP_NWEIGHTS));
    CK(cudaMemset(v, 0, sizeof(float) * ECHO_MLP_NWEIGHTS));
    CK(cudaMalloc(&act[0], sizeof(float) * B * NIN));
    for (int l = 0; l < NL; l++) {
      CK(cudaMalloc(&act[l + 1], sizeof(float) * B * LN[l]));
      CK(cudaMalloc(&dZ[l], sizeof(float) * B * LN[l]));
    }
    CK(cudaMalloc(&Y, sizeof(float) * B * 2));
    CK(cudaMalloc(&loss, sizeof(float)));
    return ECHO_OK;
  }
  // forward + backward on the batch in act[0] / Y; gradients into G
  void fwd_bwd() {
    for (int l = 0; l < NL; l++) {
      int tot = B * LN[l];
      k_linear<<<(tot + 255) / 256, 256>>>(act[l], W + WOFF[l], W + BOFF[l], act[l + 1], B, LK[l], LN[l],
                                          l < NL - 1);
    }
    cudaMemset(loss, 0, sizeof(float));
    k_loss<<<(B * 2 + 255) / 256, 256>>>(act[NL], Y, B, dZ[NL - 1], loss);
    for (int l = NL - 1; l >= 0; l--) {
      k_wgrad<<<LK[l] * LN[l], 256>>>(act[l], dZ[l], B, LK[l], LN[l], G + WOFF[l]);
      k_bgrad<<<LN[l], 256>>>(dZ[l], B, LN[l], G + BOFF[l]);
      if (l > 0) {
        int tot = B * LK[l];
        k_backact<<<(tot + 255) / 256, 256>>>(dZ[l], W + WOFF[l], act[l], B, LK[l], LN[l], dZ[l - 1]);
      }
    }
  }
};

}  // namespace

bool echo_mlp_pack(const float* W, const float* norm, std::vector<unsigned>& frag, std::vector<float>& par) {
  pack_network(W, norm, frag, par);
  return true;
}

// ---------------------------------------------------------------------------
// standalone tensor-core inference (the same mlp_warp the update kernel runs)
// ---------------------------------------------------------------------------
static __global__ void k_infer(echo::MlpDev net, const float* X, int n, float* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float f[NIN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (i < n)
    for (int j = 0; j < NIN; j++) f[j] = X[(size_t)i * NIN + j];
  float o[2];
  echo::mlp_warp(net, f, o);
  if (i < n) {
    out[(size_t)i * 2 + 0] = o[0];
    out[(size_t)i * 2 + 1] = o[1];
  }
}

extern "C" {

int echo_gpu_mlp_set(EchoCtx* c, const float* weights, const float* norm) {
  if (!c || !weights || !norm) return ECHO_ERR_ARG;
  std::vector<unsigned> frag;
  std::vector<float> par;
  pack_network(weights, norm, frag, par);
  if (!c->d_mlp_frag) {
    CK(cudaMalloc(&c->d_mlp_frag, sizeof(unsigned) * frag.size()));
    CK(cudaMalloc(&c->d_mlp_par, sizeof(float) * par.size()));
  }
  CK(cudaMemcpyAsync(c->d_mlp_frag, frag.data(), sizeof(unsigned) * frag.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_mlp_par, par.data(), sizeof(float) * par.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ECHO_OK;
}

int echo_gpu_mlp_infer(const float* weights, const float* norm, const float* X, int n, float* out) {
  if (!weights || !norm || !X || !out || n <= 0) return ECHO_ERR_ARG;
  (void)cudaGetLastError();
  std::vector<unsigned> frag;
  std::vector<float> par;
  pack_network(weights, norm, frag, par);
  unsigned* dfrag;
  float *dpar, *dX, *dout;
  CK(cudaMalloc(&dfrag, sizeof(unsigned) * frag.size()));
  CK(cudaMalloc(&dpar, sizeof(float) * par.size()));
  CK(cudaMalloc(&dX, sizeof(float) * NIN * (size_t)n));
  CK(cudaMalloc(&dout, sizeof(float) * 2 * (size_t)n));
  CK(cudaMemcpy(dfrag, frag.data(), sizeof(unsigned) * frag.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dpar, par.data(), sizeof(float) * par.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dX, X, sizeof(float) * NIN * (size_t)n, cudaMemcpyHostToDevice));
  echo::MlpDev net{dfrag, dpar};
  k_infer<<<(n + 127) / 128, 128>>>(net, dX, n, dout);
  CK(cudaGetLastError());
  CK(cudaMemcpy(out, dout, sizeof(float) * 2 * (size_t)n, cudaMemcpyDeviceToHost));
  cudaFree(dfrag);
  cudaFree(dpar);
  cudaFree(dX);
  cudaFree(dout);
  return ECHO_OK;
}

int echo_gpu_mlp_grad(const float* weights, const float* Xs, const float* Ts, int n, float* loss, float* grad) {
  if (!weights || !Xs || !Ts || n <= 0 || !loss || !grad) return ECHO_ERR_ARG;
  (void)cudaGetLastError();
  Trainer tr;
  int r = tr.alloc(n);
  if (r) return r;
  CK(cudaMemcpy(tr.W, weights, sizeof(float) * ECHO_MLP_NWEIGHTS, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(tr.act[0], Xs, sizeof(float) * NIN * (size_t)n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(tr.Y, Ts, sizeof(float) * 2 * (size_t)n, cudaMemcpyHostToDevice));
  tr.fwd_bwd();
  CK(cudaGetLastError());
  CK(cudaMemcpy(loss, tr.loss, sizeof(float), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(grad, tr.G, sizeof(float) * ECHO_MLP_NWEIGHTS, cudaMemcpyDeviceToHost));
  return ECHO_OK;
}

int echo_gpu_mlp_train(const float* X, const float* T, int n, int steps, int batch, float lr, unsigned seed,
                       float* weights_out, float* norm_out, float* loss_out, int report_every) {
  if (!X || !T || n < 2 || steps <= 0 || batch <= 0 || !weights_out || !norm_out) return ECHO_ERR_ARG;
  (void)cudaGetLastError();
  // standardisation of the raw invariants and targets
  // (a feature without spread -- E^2/U of ideal-RMHD pairs -- keeps std 1)
  double mu[NIN + 2] = {0}, sd[NIN + 2] = {0};
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < NIN; j++) mu[j] += X[(size_t)i * NIN + j];
    for (int j = 0; j < 2; j++) mu[NIN + j] += T[(size_t)i * 2 + j];
  }
  for (int j = 0; j < NIN + 2; j++) mu[j] /= n;
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < NIN; j++) sd[j] += (X[(size_t)i * NIN + j] - mu[j]) * (X[(size_t)i * NIN + j] - mu[j]);
    for (int j = 0; j < 2; j++)
      sd[NIN + j] += (T[(size_t)i * 2 + j] - mu[NIN + j]) * (T[(size_t)i * 2 + j] - mu[NIN + j]);
  }
  for (int j = 0; j < NIN + 2; j++) sd[j] = sqrt(sd[j] / n) > 1e-12 ? sqrt(sd[j] / n) : 1.0;
  for (int j = 0; j < NIN; j++) {
    norm_out[j] = (float)mu[j];
    norm_out[NIN + j] = (float)sd[j];
  }
  for (int j = 0; j < 2; j++) {
    norm_out[2 * NIN + j] = (float)mu[NIN + j];
    norm_out[2 * NIN + 2 + j] = (float)sd[NIN + j];
  }
  std::vector<float> xs((size_t)n * NIN), ts((size_t)n * 2);
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < NIN; j++) xs[(size_t)i * NIN + j] = (float)((X[(size_t)i * NIN + j] - mu[j]) / sd[j]);
    for (int j = 0; j < 2; j++)
      ts[(size_t)i * 2 + j] = (float)((T[(size_t)i * 2 + j] - mu[NIN + j]) / sd[NIN + j]);
  }
  // Glorot-uniform initial weights from a fixed-seed generator
  std::vector<float> w0(ECHO_MLP_NWEIGHTS, 0.f);
  unsigned st = seed * 2654435761u + 12345u;
  auto urand = [&]() {
    st = st * 1664525u + 1013904223u;
    return (float)((st >> 8) & 0xFFFFFF) / 16777216.f;
  };
  for (int l = 0; l < NL; l++) {
    float a = sqrtf(6.f / (float)(LK[l] + LN[l]));
    for (int i = 0; i < LK[l] * LN[l]; i++) w0[WOFF[l] + i] = (2.f * urand() - 1.f) * a;
  }
  Trainer tr;
  int r = tr.alloc(batch);
  if (r) return r;
  float *dXs, *dTs;
  CK(cudaMalloc(&dXs, sizeof(float) * xs.size()));
  CK(cudaMalloc(&dTs, sizeof(float) * ts.size()));
  CK(cudaMemcpy(dXs, xs.data(), sizeof(float) * xs.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dTs, ts.data(), sizeof(float) * ts.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(tr.W, w0.data(), sizeof(float) * ECHO_MLP_NWEIGHTS, cudaMemcpyHostToDevice));
  int nrep = 0;
  for (int s = 1; s <= steps; s++) {
    k_gather<<<(batch + 255) / 256, 256>>>(dXs, dTs, n, batch, (unsigned)s, seed, tr.act[0], tr.Y);
    tr.fwd_bwd();
    // cosine learning-rate decay to 5 % of lr
    float lrs = lr * (0.05f + 0.95f * 0.5f * (1.f + cosf(3.14159265f * (float)s / (float)steps)));
    k_adam<<<(ECHO_MLP_NWEIGHTS + 255) / 256, 256>>>(tr.W, tr.G, tr.m, tr.v, ECHO_MLP_NWEIGHTS, lrs, 0.9f, 0.999f,
                                                     1e-8f, s);
    if (loss_out && report_every > 0 && s % report_every == 0) {
      CK(cudaMemcpy(loss_out + nrep, tr.loss, sizeof(float), cudaMemcpyDeviceToHost));
      nrep++;
    }
  }
  CK(cudaGetLastError());
  CK(cudaMemcpy(weights_out, tr.W, sizeof(float) * ECHO_MLP_NWEIGHTS, cudaMemcpyDeviceToHost));
  cudaFree(dXs);
  cudaFree(dTs);
  return ECHO_OK;
}

}  // extern "C"
