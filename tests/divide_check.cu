// Test-side harness for qpb::divide and qpb::square_root, the point-wise
// step's quotient and square root, on host arrays, computed on the device.
// Built by test_gpu_divide.py with nvcc into a temporary directory.
#include <cuda_runtime.h>

#include "projection.cuh"

namespace {

__global__ void divide_kernel(const float* a, const float* b, float* q, long long n) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i < n) q[i] = qpb::divide(a[i], b[i]);
}

__global__ void sqrt_kernel(const float* a, float* q, long long n) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i < n) q[i] = qpb::square_root(a[i]);
}

}  // namespace

// q[i] = qpb::divide(a[i], b[i]) for i < n, or qpb::square_root(a[i]) when b
// is null; returns the CUDA error code.
extern "C" int divide_on_device(const float* a, const float* b, float* q, long long n) {
  float *da = nullptr, *db = nullptr, *dq = nullptr;
  const size_t bytes = static_cast<size_t>(n) * sizeof(float);
  cudaError_t e = cudaMalloc(&da, bytes);
  if (e == cudaSuccess && b) e = cudaMalloc(&db, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&dq, bytes);
  if (e == cudaSuccess) e = cudaMemcpy(da, a, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && b) e = cudaMemcpy(db, b, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int threads = 256;
    const unsigned blocks = static_cast<unsigned>((n + threads - 1) / threads);
    if (b) {
      divide_kernel<<<blocks, threads>>>(da, db, dq, n);
    } else {
      sqrt_kernel<<<blocks, threads>>>(da, dq, n);
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(q, dq, bytes, cudaMemcpyDeviceToHost);
  cudaFree(da);
  cudaFree(db);
  cudaFree(dq);
  return static_cast<int>(e);
}
