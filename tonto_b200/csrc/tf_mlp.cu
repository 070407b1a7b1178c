// tf_mlp.cu — training and inference kernels of the learned initial-density
// network (an MLP with SiLU activations, FP32 weights and activations).
//
//   tf_mlp_gemm     C = op(A) op(B) (+ bias) (+ SiLU), smem-tiled 64x64x16,
//                   with the pre-activation optionally kept for the backward pass
//   tf_mlp_silu_bwd dZ = dA * silu'(Z)
//   tf_mlp_colsum   db = sum over rows of dZ (bias gradient)
//   tf_mlp_mse      weighted squared error and its gradient
//   tf_mlp_adam     Adam update (bias-corrected)
//
// All pointers are device pointers; every call is asynchronous on `stream`.
// The network has no counterpart in Tonto: it only proposes an initial density.
#include <cuda_runtime.h>
#include <math.h>

#include "../../include/tontofock_guess.h"

namespace {

constexpr int TM = 64, TN = 64, TK = 16;

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// C[M x N] = sum_k A(i,k) B(k,j); A(i,k) = A[i*sai + k*sak], B(k,j) = B[k*sbk + j*sbj].
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float* __restrict__ A, long sai, long sak,
                                              const float* __restrict__ B, long sbk, long sbj,
                                              const float* __restrict__ bias, int act, float* __restrict__ Zout,
                                              float* __restrict__ C, float beta) {
  __shared__ float As[TK][TM + 4];
  __shared__ float Bs[TK][TN + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int i0 = blockIdx.y * TM, j0 = blockIdx.x * TN;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int q = threadIdx.x; q < TM * TK; q += 256) {
      const int ii = q / TK, kk = q % TK;
      const int i = i0 + ii, k = k0 + kk;
      As[kk][ii] = (i < M && k < K) ? A[i * sai + k * sak] : 0.0f;
    }
    for (int q = threadIdx.x; q < TN * TK; q += 256) {
      const int kk = q / TN, jj = q % TN;
      const int k = k0 + kk, j = j0 + jj;
      Bs[kk][jj] = (k < K && j < N) ? B[k * sbk + j * sbj] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[kk][ty * 4 + r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = Bs[kk][tx * 4 + c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int i = i0 + ty * 4 + r, j = j0 + tx * 4 + c;
      if (i >= M || j >= N) continue;
      float z = acc[r][c] + (bias ? bias[j] : 0.0f);
      if (beta != 0.0f) z += beta * C[(long)i * N + j];
      if (Zout) Zout[(long)i * N + j] = z;
      C[(long)i * N + j] = act ? silu(z) : z;
    }
}

__global__ void k_silu_bwd(long n, const float* __restrict__ dA, const float* __restrict__ Z, float* __restrict__ dZ) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dZ[t] = dA[t] * silu_grad(Z[t]);
}

// db[j] = sum_i dZ[i][j]: one block per 32 columns, threads over rows (deterministic order)
__global__ void k_colsum(int M, int N, const float* __restrict__ dZ, float* __restrict__ db) {
  __shared__ float part[8][33];
  const int j = blockIdx.x * 32 + (threadIdx.x & 31), r = threadIdx.x >> 5;
  float s = 0.0f;
  if (j < N)
    for (int i = r; i < M; i += 8) s += dZ[(long)i * N + j];
  part[r][threadIdx.x & 31] = s;
  __syncthreads();
  if (r == 0 && j < N) {
    float t = 0.0f;
    for (int q = 0; q < 8; ++q) t += part[q][threadIdx.x & 31];
    db[j] = t;
  }
}

// loss = sum_i w_i * sum_j (Y - T)^2 / norm;  dY = 2 w (Y - T) / norm.  Per-block
// partial losses go to loss_part[blockIdx.x] (summed by the caller).
__global__ void k_mse(int M, int N, const float* __restrict__ Y, const float* __restrict__ T,
                      const float* __restrict__ w, float inv_norm, float* __restrict__ dY,
                      float* __restrict__ loss_part) {
  __shared__ float red[256];
  const long n = (long)M * N;
  float s = 0.0f;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const float wi = w ? w[t / N] : 1.0f;
    const float d = Y[t] - T[t];
    s += wi * d * d;
    dY[t] = 2.0f * wi * d * inv_norm;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0] * inv_norm;
}

__global__ void k_adam(long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                       float wd) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t] + wd * p[t];
  const float mt = b1 * m[t] + (1.0f - b1) * gt;
  const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

}  // namespace

extern "C" {

int tf_mlp_gemm(int M, int N, int K, const float* A, long sai, long sak, const float* B, long sbk, long sbj,
                const float* bias, int act, float* Zout, float* C, float beta, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return -1;
  dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  k_gemm<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(M, N, K, A, sai, sak, B, sbk, sbj, bias, act, Zout,
                                                             C, beta);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int tf_mlp_silu_bwd(long n, const float* dA, const float* Z, float* dZ, void* stream) {
  if (n <= 0) return -1;
  k_silu_bwd<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, dA, Z, dZ);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int tf_mlp_colsum(int M, int N, const float* dZ, float* db, void* stream) {
  if (M <= 0 || N <= 0) return -1;
  k_colsum<<<(N + 31) / 32, 256, 0, static_cast<cudaStream_t>(stream)>>>(M, N, dZ, db);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int tf_mlp_mse(int M, int N, const float* Y, const float* T, const float* w, float inv_norm, float* dY,
               float* loss_part, int n_blocks, void* stream) {
  if (M <= 0 || N <= 0 || n_blocks <= 0) return -1;
  k_mse<<<n_blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(M, N, Y, T, w, inv_norm, dY, loss_part);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int tf_mlp_adam(long n, float* p, const float* g, float* m, float* v, float lr, float beta1, float beta2, float eps,
                int step, float weight_decay, void* stream) {
  if (n <= 0 || step < 1) return -1;
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  k_adam<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, p, g, m, v, lr, beta1,
                                                                                     beta2, eps, c1, c2,
                                                                                     weight_decay);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // extern "C"
