// align_noalloc.cu -- stormgpu_align_noalloc: the full banded alignment with traceback of one
// read against n windows (the computation of stormgpu_align), for callers that cannot
// allocate device memory.
//
// Who needs it: a caller whose device memory belongs to another allocator -- a framework's
// caching allocator or a pool reserved at start-up, with no room outside it, where a
// cudaMalloc would fail or break the memory budget -- or a latency-bound caller for whom the
// implicit device-wide synchronisation of cudaMalloc / cudaFree would stall the work on its
// other streams.  Such a caller allocates its inputs and outputs itself; the working memory
// of the alignment kernel (two traceback direction bits per band cell, plus per-window
// bookkeeping) then has to come from somewhere that is not an allocation.
//
// It comes from g_noalloc_scratch below: one file-scope device array of kNoAllocScratchBytes
// (8 MiB) that every GPU which loads this library holds until the process exits.  In host
// code the array's name is only a host-side stand-in for it; its device address is obtained
// with cudaGetSymbolAddress, with that device current, at the start of every call (the first
// call on a device also loads the module there).  Every call shares the array and it keeps
// the last call's contents: what must start at zero (the error count, the per-window read
// indices) is cleared by each call.
#include <cstring>

#include "map_kernels.cuh"

namespace {

using namespace sg;

constexpr int64_t kNoAllocScratchBytes = 8ll << 20;
static_assert(kNoAllocScratchBytes == STORMGPU_NOALLOC_SCRATCH_BYTES, "scratch size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Layout of the scratch for a call with n windows (byte offsets, all 256-aligned):
//   [0, 4)      number of windows outside the genome (uint32)
//   [4, 6)      read length (int16)
//   [256, ...)  per-window read index (int32, all 0), then per-window diagonal (int32)
//   [dir, ...)  traceback direction words, L * words_per_row * n uint32
constexpr int64_t kHeaderBytes = 256;
inline int64_t round256(int64_t x) { return (x + 255) & ~255LL; }

// Device address of the scratch on the current device.  cudaGetSymbolAddress allocates
// nothing; it is asked on every call rather than cached, so that an address never outlives
// the module it came from (a device reset or a primary-context release reloads the module).
int scratch_address(int dev, unsigned char** out) {
  unsigned char* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr) {
    sg_set_error("stormgpu_align_noalloc: cudaGetSymbolAddress of the scratch array failed on device %d: %s",
                 dev, cudaGetErrorString(e));
    return STORMGPU_ECUDA;
  }
  *out = ptr;
  return 0;
}

// Per window: read index 0 and diagonal win + I; a window that does not lie inside the
// genome ([win, win + L + 2I) within [0, n_codes)) is counted and aligned at window 0
// instead, so that no access leaves the caller's buffers.
__global__ void noalloc_prep_kernel(const int32_t* __restrict__ win, int64_t n, int I, int L, int64_t n_codes,
                                    int32_t* __restrict__ p_read, int32_t* __restrict__ p_diag,
                                    int16_t* __restrict__ len, unsigned* __restrict__ bad) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t w = win[t];
    const bool ok = w >= 0 && w + L + 2 * (int64_t)I <= n_codes;
    p_read[t] = 0;
    p_diag[t] = (int32_t)((ok ? w : 0) + I);
    if (!ok) atomicAdd(bad, 1u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *len = (int16_t)L;
}

}  // namespace

extern "C" int stormgpu_align_noalloc(const stormgpu_params* params, const uint8_t* read, const uint8_t* levels,
                                      int read_len, const uint8_t* genome, const uint8_t* mask, int64_t n_codes,
                                      const int32_t* win, int64_t n, int32_t* score, int32_t* bound, int16_t* best,
                                      int32_t* tb_len, uint8_t* tb, int64_t tb_stride, void* stream) {
  if (!params || read_len <= 0 || read_len > STORMGPU_MAX_READ_LEN || n < 0 || params->allowed_indels < 0 ||
      params->allowed_indels > STORMGPU_MAX_INDELS) {
    sg_set_error("stormgpu_align_noalloc: bad arguments");
    return STORMGPU_EINVAL;
  }
  const int I = params->allowed_indels;
  if (tb_stride < (read_len + I + 1) / 2) {
    sg_set_error("stormgpu_align_noalloc: tb_stride %lld < %d", (long long)tb_stride, (read_len + I + 1) / 2);
    return STORMGPU_EINVAL;
  }
  if (n_codes < read_len + 2 * (int64_t)I) {
    sg_set_error("stormgpu_align_noalloc: genome of %lld codes shorter than one window (%lld codes)",
                 (long long)n_codes, (long long)(read_len + 2 * (int64_t)I));
    return STORMGPU_EINVAL;
  }
  const int BW = 2 * I + 1;
  const int wpr = (2 * BW + 31) / 32 + (params->colour ? (BW + 31) / 32 : 0);
  const int64_t off_read = kHeaderBytes;
  const int64_t off_diag = off_read + round256(4 * n);
  const int64_t off_dir = off_diag + round256(4 * n);
  const int64_t need = off_dir + 4 * (int64_t)read_len * wpr * n;
  if (need > kNoAllocScratchBytes) {
    sg_set_error("stormgpu_align_noalloc: %lld windows of a %d-code read with -i %d need %lld bytes of scratch, "
                 "more than its %lld bytes; split the windows over several calls",
                 (long long)n, read_len, I, (long long)need, (long long)kNoAllocScratchBytes);
    return STORMGPU_EINVAL;
  }
  if (!read || !genome || !mask || (n > 0 && (!win || !score || !bound || !best || !tb_len || !tb))) {
    sg_set_error("stormgpu_align_noalloc: null buffer");
    return STORMGPU_EINVAL;
  }
  if (n == 0) return 0;
  int dev = 0;
  SG_CUDA(cudaGetDevice(&dev));
  unsigned char* scr = nullptr;
  if (const int rc = scratch_address(dev, &scr)) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  unsigned* bad = reinterpret_cast<unsigned*>(scr);
  int16_t* len = reinterpret_cast<int16_t*>(scr + 4);
  int32_t* p_read = reinterpret_cast<int32_t*>(scr + off_read);
  int32_t* p_diag = reinterpret_cast<int32_t*>(scr + off_diag);
  SG_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), st));
  SG_CUDA(cudaMemsetAsync(tb, 0, (size_t)(tb_stride * n), st));
  int64_t blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  noalloc_prep_kernel<<<(unsigned)blocks, 256, 0, st>>>(win, n, I, read_len, n_codes, p_read, p_diag, len, bad);
  SG_CUDA(cudaGetLastError());

  ScoreParams sp = make_score_params(*params);
  sp.Is = 1 << 28;            // window = diag - I exactly
  sp.min_score = -(1 << 29);  // always trace back
  sp.packed = 0;                // every cell exact: no floor
  const int64_t rb = (read_len + 3) / 4;
  ReadsDev rd{1, read, rb, levels, rb, len};
  PassBuffers pb;
  memset(&pb, 0, sizeof(pb));
  pb.p_read = p_read;
  pb.p_diag = p_diag;
  pb.a_score = score;
  pb.a_bound = bound;
  pb.a_pos = best;
  pb.a_tblen = tb_len;
  pb.a_tb = tb;
  pb.tbs = tb_stride;
  pb.a_scratch = reinterpret_cast<uint32_t*>(scr + off_dir);
  pb.scratch_words = (int64_t)read_len * wpr * n;
  launch_align(rd, sp, genome, mask, 0, n, pb, st);
  SG_CUDA(cudaGetLastError());

  unsigned nbad = 0;
  SG_CUDA(cudaMemcpyAsync(&nbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  if (nbad) {
    sg_set_error("stormgpu_align_noalloc: %u of %lld windows not inside the %lld-code genome", nbad, (long long)n,
                 (long long)n_codes);
    return STORMGPU_EINVAL;
  }
  return 0;
}
