// Test helper (not part of the library): compares the Newton-Raphson reciprocal
// and reciprocal square root of the kernels with IEEE division and square root.
#include "tf_device.cuh"

__global__ void k_check(const double* x, int n, double* err_rcp, double* err_rsqrt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = x[i];
  const double r = 1.0 / v, q = 1.0 / sqrt(v);
  err_rcp[i] = fabs(tf::rcp_nr(v) - r) / r;
  err_rsqrt[i] = fabs(tf::rsqrt_nr(v) - q) / q;
}

extern "C" int fast_math_check(const double* x, int n, double* err_rcp, double* err_rsqrt) {
  double *dx, *dr, *dq;
  if (cudaMalloc(&dx, n * sizeof(double)) || cudaMalloc(&dr, n * sizeof(double)) ||
      cudaMalloc(&dq, n * sizeof(double)))
    return 1;
  cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice);
  k_check<<<(n + 255) / 256, 256>>>(dx, n, dr, dq);
  cudaMemcpy(err_rcp, dr, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(err_rsqrt, dq, n * sizeof(double), cudaMemcpyDeviceToHost);
  const int rc = cudaGetLastError() != cudaSuccess;
  cudaFree(dx); cudaFree(dr); cudaFree(dq);
  return rc;
}
