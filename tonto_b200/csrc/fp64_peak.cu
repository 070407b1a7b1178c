// fp64_peak.cu — measures the FP64 FMA-pipe throughput of the current GPU with a
// register-resident chain of fused multiply-adds (8 independent chains per
// thread, grid = 8 blocks of 256 threads per SM).  Used as the roofline
// denominator for the FP64 Rys kernels.
#include <cuda_runtime.h>

__global__ void k_fma_loop(double* out, int iters, double b, double c) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
  double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
      a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
  }
  const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 1.2345) out[blockIdx.x * blockDim.x + threadIdx.x] = s;   // keeps the chain live
}

__global__ void k_fma_loop_f32(float* out, int iters, float b, float c) {
  float a[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = threadIdx.x * 1e-6f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int k = 0; k < 16; ++k) a[k] = fmaf(a[k], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += a[k];
  if (s == 1.2345f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

extern "C" int tf_peak_fma(int device, int fp32, double* tflops, double* ms) {
  if (cudaSetDevice(device) != cudaSuccess) return -1;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  const int threads = 256, blocks = nsm * 8, iters = 4096;
  void* out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * threads * 8) != cudaSuccess) return -2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    if (fp32) k_fma_loop_f32<<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
    else k_fma_loop<<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-9);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (rep > 0 && t < best) best = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -3;
  const double fma_per_thread = fp32 ? (double)iters * 8 * 16 : (double)iters * 16 * 8;
  *tflops = 2.0 * fma_per_thread * blocks * threads / (best * 1e-3) / 1e12;
  *ms = best;
  return 0;
}
