// intpeak.cu -- the roofline denominator of the banded filter, measured on this GPU: every
// thread runs 16 independent register-resident copies of one step of the packed 16-bit filter
// recurrence (filter_core.cuh), with no memory traffic, so that the figure is the chip's rate
// for that exact instruction mix rather than a datasheet number.
//
// Per copy and step (one register = two 16-bit cells): a gap subtraction and an add-max (P), a
// three-way max (I), a subtraction and a byte permute (score), an add-max (M), and half of a
// three-way max (running maximum): 6.5 32-bit lane instructions per two cells.
#include "common.cuh"
#include "filter_core.cuh"

namespace {

__global__ void filter_mix_kernel(int iters, uint32_t seed, uint32_t* out) {
  uint32_t M1[16], M2[16], I1[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    M1[k] = (seed + 977u * k + threadIdx.x) & 0x00ff00ffu;
    M2[k] = (seed * 3u + 131u * k) & 0x00ff00ffu;
    I1[k] = (seed ^ (k * 0x01010101u)) & 0x00ff00ffu;
  }
  const uint32_t NFE = (uint32_t)(uint16_t)(-(int)(seed & 3u)) * 0x10001u, CFO = ((seed >> 2) & 7u) * 0x10001u;
  const uint32_t TLO = seed * 0x9E3779B9u, THI = TLO ^ 0x5A5A5A5Au;
  uint32_t mx0 = 0, mx1 = 0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint32_t p = __viaddmax_s16x2(I1[k], NFE, M1[k] - CFO);
      const uint32_t in = __vimax3_s16x2(p, I1[(k + 1) & 15], sg::kFBB);
      const uint32_t sc = sg::prmt(TLO, THI, M1[k] - M2[k]);
      const uint32_t mn = __viaddmax_s16x2(M2[k], sc, in);
      M2[k] = M1[k];
      M1[k] = mn;
      I1[k] = in;
    }
#pragma unroll
    for (int k = 0; k < 16; k += 4) {
      mx0 = __vimax3_s16x2(mx0, M1[k], M1[k + 1]);
      mx1 = __vimax3_s16x2(mx1, M1[k + 2], M1[k + 3]);
    }
  }
  uint32_t s = mx0 ^ mx1;
#pragma unroll
  for (int k = 0; k < 16; ++k) s ^= M1[k] ^ I1[k];
  if (s == 0x7fffffffu) out[0] = s;  // keep the work alive
}

}  // namespace

// 32-bit lane instructions of the filter recurrence per second (6.5 per register step).
extern "C" int stormgpu_filter_peak(int device, double* ops_per_s, double* ms) {
  SG_CUDA(cudaSetDevice(device));
  int sms = 0;
  SG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  uint32_t* d;
  SG_CUDA(cudaMalloc(&d, sizeof(uint32_t)));
  cudaEvent_t e0, e1;
  SG_CUDA(cudaEventCreate(&e0));
  SG_CUDA(cudaEventCreate(&e1));
  const int blocks = sms * 8, threads = 256, iters = 4000;
  filter_mix_kernel<<<blocks, threads>>>(100, 1u, d);  // warm-up
  SG_CUDA(cudaEventRecord(e0));
  filter_mix_kernel<<<blocks, threads>>>(iters, 2u, d);
  SG_CUDA(cudaEventRecord(e1));
  SG_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  SG_CUDA(cudaEventElapsedTime(&t, e0, e1));
  *ms = t;
  *ops_per_s = (double)blocks * threads * iters * (16 * 6 + 8) / (t * 1e-3);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  return 0;
}
