// Order-selection network: a 3-layer perceptron 12 -> 64 -> 64 -> 6
// (ReLU, ReLU, logits over interpolation orders 3..8), trained and run by
// the kernels below.  Parameters are one flat FP32 array in the order
//   W1 (64 x 12, row-major), b1 (64), W2 (64 x 64), b2 (64), W3 (6 x 64), b3 (6)
// and, for inference, a BF16 copy of the same array.  Samples are rows of
// X (n x 12, row-major); activations are rows of H1, H2 (n x 64) and
// logits (n x 6).
//
// Training (FP32): forward, softmax cross-entropy with per-sample weights,
// backward through small tiled GEMMs (one kernel, transposes by strides),
// per-parameter Adam with decoupled weight decay.  Inference: BF16 weights
// in shared memory, FP32 accumulation, one thread per sample.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/defmm_b200.h"

namespace {

constexpr int NIN = DEFMM_MLP_IN, NH = DEFMM_MLP_HIDDEN, NOUT = DEFMM_MLP_OUT;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NIN, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NOUT * NH, NPARAM = OFF_B3 + NOUT;
static_assert(NPARAM == DEFMM_MLP_PARAMS, "parameter count");

// C[m][n] = sum_k A(m, k) B(k, n) with A(m, k) = A[m * as0 + k * as1] and
// B(k, n) = B[k * bs0 + n * bs1] (any transposes by strides); C row-major
// with leading dimension ldc.  16 x 16 output tiles, K in steps of 16
// through shared memory.
__global__ void k_gemm(int M, int N, int K, const float* __restrict__ A, int64_t as0, int64_t as1,
                       const float* __restrict__ B, int64_t bs0, int64_t bs1, float* __restrict__ C, int64_t ldc) {
  __shared__ float As[16][17], Bs[16][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m = blockIdx.y * 16 + ty, n = blockIdx.x * 16 + tx;
  float acc = 0.f;
  for (int k0 = 0; k0 < K; k0 += 16) {
    const int ka = k0 + tx, kb = k0 + ty;
    As[ty][tx] = (m < M && ka < K) ? A[m * as0 + ka * as1] : 0.f;
    Bs[ty][tx] = (kb < K && n < N) ? B[kb * bs0 + n * bs1] : 0.f;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; k++) acc = fmaf(As[ty][k], Bs[k][tx], acc);
    __syncthreads();
  }
  if (m < M && n < N) C[m * ldc + n] = acc;
}

void gemm(int M, int N, int K, const float* A, int64_t as0, int64_t as1, const float* B, int64_t bs0, int64_t bs1,
          float* C, int64_t ldc, cudaStream_t s) {
  dim3 grid((N + 15) / 16, (M + 15) / 16);
  k_gemm<<<grid, 256, 0, s>>>(M, N, K, A, as0, as1, B, bs0, bs1, C, ldc);
}

// Z[i][j] += b[j]; optionally Z = max(Z, 0)
__global__ void k_bias_act(int64_t n, int width, const float* __restrict__ b, float* __restrict__ Z, int relu) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * width) return;
  const float v = Z[i] + b[i % width];
  Z[i] = (relu && v < 0.f) ? 0.f : v;
}

// softmax cross-entropy: G = w_i (softmax(logits_i) - onehot(y_i)) / sum w;
// loss += w_i (-log softmax_y) / sum w  (atomically)
__global__ void k_xent(int64_t n, const float* __restrict__ logits, const int32_t* __restrict__ y,
                       const float* __restrict__ w, float inv_wsum, float* __restrict__ G, float* __restrict__ loss) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* z = logits + i * NOUT;
  float mx = z[0];
  for (int c = 1; c < NOUT; c++) mx = fmaxf(mx, z[c]);
  float e[NOUT], s = 0.f;
  for (int c = 0; c < NOUT; c++) {
    e[c] = expf(z[c] - mx);
    s += e[c];
  }
  const float wi = (w ? w[i] : 1.f) * inv_wsum;
  const int yi = y[i];
  for (int c = 0; c < NOUT; c++) G[i * NOUT + c] = wi * (e[c] / s - (c == yi ? 1.f : 0.f));
  atomicAdd(loss, wi * (logf(s) - (z[yi] - mx)));
}

// D[i][j] = 0 where H[i][j] <= 0  (ReLU derivative through the stored activation)
__global__ void k_relu_back(int64_t count, const float* __restrict__ H, float* __restrict__ D) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < count && !(H[i] > 0.f)) D[i] = 0.f;
}

// db[j] = sum_i D[i][j]; one block of 256 threads per column
__global__ void k_colsum(int64_t n, int width, const float* __restrict__ D, float* __restrict__ db) {
  const int j = blockIdx.x;
  float s = 0.f;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += D[i * width + j];
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[j] = red[0];
}

// Adam with decoupled weight decay wd (applied to every parameter)
__global__ void k_adam(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float wd, float b1, float b2, float c1, float c2, float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i]);
}

__global__ void k_to_bf16(int n, const float* __restrict__ p, __nv_bfloat16* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2bfloat16_rn(p[i]);
}

// one thread per sample; BF16 parameters staged in shared memory
__global__ void __launch_bounds__(128) k_infer_bf16(int64_t n, const __nv_bfloat16* __restrict__ P,
                                                    const float* __restrict__ X, float* __restrict__ out) {
  __shared__ __nv_bfloat16 sp[NPARAM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) sp[i] = P[i];
  __syncthreads();
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  float x[NIN], h1[NH], h2[NH];
#pragma unroll
  for (int k = 0; k < NIN; k++) x[k] = X[s * NIN + k];
  for (int j = 0; j < NH; j++) {
    float a = __bfloat162float(sp[OFF_B1 + j]);
#pragma unroll
    for (int k = 0; k < NIN; k++) a = fmaf(__bfloat162float(sp[OFF_W1 + j * NIN + k]), x[k], a);
    h1[j] = fmaxf(a, 0.f);
  }
  for (int j = 0; j < NH; j++) {
    float a = __bfloat162float(sp[OFF_B2 + j]);
    for (int k = 0; k < NH; k++) a = fmaf(__bfloat162float(sp[OFF_W2 + j * NH + k]), h1[k], a);
    h2[j] = fmaxf(a, 0.f);
  }
  for (int c = 0; c < NOUT; c++) {
    float a = __bfloat162float(sp[OFF_B3 + c]);
    for (int k = 0; k < NH; k++) a = fmaf(__bfloat162float(sp[OFF_W3 + c * NH + k]), h2[k], a);
    out[s * NOUT + c] = a;
  }
}

int status(cudaError_t e) {
  if (e == cudaSuccess) return 0;
  cudaGetLastError();
  return DEFMM_ERR_CUDA;
}

int blocks(int64_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

extern "C" {

int defmm_mlp_forward(const float* params, const float* X, int64_t n, float* H1, float* H2, float* logits,
                      void* stream) {
  if (!params || !X || !H1 || !H2 || !logits || n < 1 || n > (1 << 30)) return DEFMM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  // H1 = relu(X W1^T + b1): A = X (n x 12), B(k, j) = W1[j][k]
  gemm((int)n, NH, NIN, X, NIN, 1, params + OFF_W1, 1, NIN, H1, NH, s);
  k_bias_act<<<blocks(n * NH, 256), 256, 0, s>>>(n, NH, params + OFF_B1, H1, 1);
  gemm((int)n, NH, NH, H1, NH, 1, params + OFF_W2, 1, NH, H2, NH, s);
  k_bias_act<<<blocks(n * NH, 256), 256, 0, s>>>(n, NH, params + OFF_B2, H2, 1);
  gemm((int)n, NOUT, NH, H2, NH, 1, params + OFF_W3, 1, NH, logits, NOUT, s);
  k_bias_act<<<blocks(n * NOUT, 256), 256, 0, s>>>(n, NOUT, params + OFF_B3, logits, 0);
  return status(cudaGetLastError());
}

int defmm_mlp_backward(const float* params, const float* X, const float* H1, const float* H2, const float* logits,
                       const int32_t* y, const float* w, float wsum, int64_t n, float* grads, float* loss,
                       float* scratch, void* stream) {
  if (!params || !X || !H1 || !H2 || !logits || !y || !grads || !loss || !scratch || n < 1 || n > (1 << 30) ||
      !(wsum > 0.f))
    return DEFMM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  float* G3 = scratch;        // n x 6
  float* D2 = G3 + n * NOUT;  // n x 64
  float* D1 = D2 + n * NH;    // n x 64
  cudaMemsetAsync(loss, 0, sizeof(float), s);
  k_xent<<<blocks(n, 256), 256, 0, s>>>(n, logits, y, w, 1.f / wsum, G3, loss);
  // dW3 = G3^T H2 (6 x 64), db3 = column sums of G3
  gemm(NOUT, NH, (int)n, G3, 1, NOUT, H2, NH, 1, grads + OFF_W3, NH, s);
  k_colsum<<<NOUT, 256, 0, s>>>(n, NOUT, G3, grads + OFF_B3);
  // D2 = (G3 W3) o [H2 > 0]
  gemm((int)n, NH, NOUT, G3, NOUT, 1, params + OFF_W3, NH, 1, D2, NH, s);
  k_relu_back<<<blocks(n * NH, 256), 256, 0, s>>>(n * NH, H2, D2);
  gemm(NH, NH, (int)n, D2, 1, NH, H1, NH, 1, grads + OFF_W2, NH, s);
  k_colsum<<<NH, 256, 0, s>>>(n, NH, D2, grads + OFF_B2);
  // D1 = (D2 W2) o [H1 > 0]
  gemm((int)n, NH, NH, D2, NH, 1, params + OFF_W2, NH, 1, D1, NH, s);
  k_relu_back<<<blocks(n * NH, 256), 256, 0, s>>>(n * NH, H1, D1);
  gemm(NH, NIN, (int)n, D1, 1, NH, X, NIN, 1, grads + OFF_W1, NIN, s);
  k_colsum<<<NH, 256, 0, s>>>(n, NH, D1, grads + OFF_B1);
  return status(cudaGetLastError());
}

int defmm_mlp_adam(float* params, const float* grads, float* m, float* v, int64_t step, float lr, float wd,
                   void* stream) {
  if (!params || !grads || !m || !v || step < 1 || !(lr > 0.f) || !(wd >= 0.f)) return DEFMM_ERR_ARG;
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.f, c2 = 1.f;
  for (int64_t i = 0; i < step && i < 10000; i++) {
    c1 *= b1;
    c2 *= b2;
  }
  k_adam<<<blocks(NPARAM, 256), 256, 0, (cudaStream_t)stream>>>(NPARAM, params, grads, m, v, lr, wd, b1, b2,
                                                                  1.f - c1, 1.f - c2, 1e-8f);
  return status(cudaGetLastError());
}

int defmm_mlp_to_bf16(const float* params, uint16_t* out, void* stream) {
  if (!params || !out) return DEFMM_ERR_ARG;
  k_to_bf16<<<blocks(NPARAM, 256), 256, 0, (cudaStream_t)stream>>>(NPARAM, params,
                                                                    reinterpret_cast<__nv_bfloat16*>(out));
  return status(cudaGetLastError());
}

int defmm_mlp_infer_bf16(const uint16_t* params_bf16, const float* X, int64_t n, float* logits, void* stream) {
  if (!params_bf16 || !X || !logits || n < 1) return DEFMM_ERR_ARG;
  k_infer_bf16<<<blocks(n, 128), 128, 0, (cudaStream_t)stream>>>(
      n, reinterpret_cast<const __nv_bfloat16*>(params_bf16), X, logits);
  return status(cudaGetLastError());
}

}  // extern "C"
