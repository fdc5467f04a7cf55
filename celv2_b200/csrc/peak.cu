// peak.cu: the INT32 ALU throughput of the GPU, measured in the run that reports a roofline
// against it. The decision kernels are integer-ALU bound (SAD, Hadamard, compares); their roofline
// denominator is this measured rate, taken like the measured HBM and GEMM peaks: a dependent chain
// of 32-bit adds and logic ops per thread, eight independent chains, grid of 8 CTAs per SM.
#include <cuda_runtime.h>

#include <cstdint>

namespace celv2cu {

__global__ void k_int_chain(uint32_t* out, int iters) {
  uint32_t v[8];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = threadIdx.x + i * 977u;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 16; k++)
#pragma unroll
      for (int i = 0; i < 8; i++) v[i] = v[i] + (v[(i + 1) & 7] ^ (uint32_t)k);
  }
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += v[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Integer ops per second (an add and an xor per element step), best of 3 timed runs.
cudaError_t measure_int_peak(int device, double* ops_per_s) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return e;
  cudaDeviceProp p;
  if ((e = cudaGetDeviceProperties(&p, device)) != cudaSuccess) return e;
  const int blocks = p.multiProcessorCount * 8, threads = 256, iters = 2000;
  uint32_t* out = nullptr;
  if ((e = cudaMalloc(&out, (size_t)blocks * threads * sizeof(uint32_t))) != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 0;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(a);
    k_int_chain<<<blocks, threads>>>(out, iters);
    cudaEventRecord(b);
    if ((e = cudaEventSynchronize(b)) != cudaSuccess) break;
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    const double ops = (double)blocks * threads * iters * 16 * 8 * 2;
    if (rep > 0 && ops / (ms * 1e-3) > best) best = ops / (ms * 1e-3);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  *ops_per_s = best;
  return e;
}

}  // namespace celv2cu
