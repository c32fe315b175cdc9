// intpeak.cu -- integer-pipe peak of this GPU, measured: every thread runs 16 independent
// chains of add + max (the instruction mix of the banded filter), so that the figure is the
// chip's issue rate for those 32-bit integer operations, not a datasheet number.
#include "common.cuh"

namespace {

__global__ void intpeak_kernel(int iters, int seed, int* out) {
  int a[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = seed + k * 7 + threadIdx.x;
  const int b = seed * 3 + 1, c = seed ^ 0x55;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a[k] = a[k] + b;          // IADD
      a[k] = max(a[k], c);      // IMNMX
    }
  }
  int s = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) s ^= a[k];
  if (s == 0x7fffffff) out[0] = s;  // keep the work alive
}

}  // namespace

// Sustained 32-bit integer add/max lane-operations per second (ops counted per thread).
extern "C" int stormgpu_int_peak(int device, double* ops_per_s, double* ms) {
  SG_CUDA(cudaSetDevice(device));
  int sms = 0;
  SG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  int* d;
  SG_CUDA(cudaMalloc(&d, sizeof(int)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256, iters = 20000;
  intpeak_kernel<<<blocks, threads>>>(100, 1, d);  // warm-up
  cudaEventRecord(e0);
  intpeak_kernel<<<blocks, threads>>>(iters, 2, d);
  cudaEventRecord(e1);
  SG_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  *ms = t;
  *ops_per_s = (double)blocks * threads * iters * 16 * 2 / (t * 1e-3);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  return 0;
}
