// genome_map.cu -- the greedy placement of the mapping without -M (-G, genome_map.c:187-214):
// every read with an alignment goes to the start of its rank-0 alignment, and the SAM lists
// positions in order with the reads of one position in read order
// (genome_map.c:551-796).  Here: one key per read (its global position, or "not placed"), a
// stable radix sort of (key, read), the placed prefix returned.  The stable sort is what keeps
// read order within a position.
#include <cstring>

#include "context.cuh"
#include "radix.cuh"

namespace {

using namespace sg;

constexpr uint32_t kNotPlaced = 0xffffffffu;

__global__ void greedy_keys_kernel(int64_t n, const stormgpu_hit* __restrict__ hits, const uint8_t* __restrict__ mapped,
                                   const uint32_t* __restrict__ base, int uniqueness_threshold,
                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                   unsigned long long* __restrict__ placed) {
  unsigned long long cnt = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const stormgpu_hit h0 = hits[r * 4], h1 = hits[r * 4 + 1];
    const bool ok = mapped[r] && h0.ref_start != STORMGPU_UNMAPPED &&
                    (uniqueness_threshold <= 0 || h0.score - h1.score >= uniqueness_threshold);
    keys[r] = ok ? base[h0.ref_id] + (uint32_t)h0.ref_start : kNotPlaced;
    vals[r] = (uint32_t)r;
    cnt += ok ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(placed, cnt);
}

}  // namespace

extern "C" int stormgpu_genome_map_greedy(stormgpu_ctx* c, int32_t uniqueness_threshold, int32_t* order,
                                          int64_t* n_placed) {
  if (!c || !order || !n_placed) { sg_set_error("stormgpu_genome_map_greedy: null argument"); return STORMGPU_EINVAL; }
  if (c->last_n < 0) { sg_set_error("stormgpu_genome_map_greedy: no stormgpu_map call yet"); return STORMGPU_ESTATE; }
  SG_CUDA(cudaSetDevice(c->p.device));
  const int64_t n = c->last_n;
  *n_placed = 0;
  if (n == 0) return 0;
  // global position of every sequence's code 0; every sequence has size + 1 positions
  std::vector<uint32_t> base(c->refs.size() + 1, 0);
  uint64_t acc = 0;
  for (size_t s = 0; s < c->refs.size(); ++s) {
    base[s] = (uint32_t)acc;
    acc += (uint64_t)c->refs[s].n + 1;
  }
  if (acc >= kNotPlaced || n >= (int64_t)kNotPlaced) {
    sg_set_error("stormgpu_genome_map_greedy: more than 2^32 - 1 reference positions or reads");
    return STORMGPU_EINVAL;
  }
  cudaStream_t st = c->st;
  if (c->gm_k0.grow(n) || c->gm_v0.grow(n) || c->gm_k1.grow(n) || c->gm_v1.grow(n) ||
      c->gm_tmp.grow(radix_tmp_bytes(n) / 4 + 16) || c->gm_base.grow((int64_t)base.size()) || c->counters.grow(16))
    return STORMGPU_ENOMEM;
  SG_CUDA(cudaMemcpyAsync(c->gm_base.p, base.data(), sizeof(uint32_t) * base.size(), cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long), st));
  int64_t blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  greedy_keys_kernel<<<(unsigned)blocks, 256, 0, st>>>(n, c->hits.p, c->mapped.p, c->gm_base.p, uniqueness_threshold,
                                                        c->gm_k0.p, c->gm_v0.p, c->counters.p);
  SG_CUDA(cudaGetLastError());
  const int which = radix_sort_pairs(c->gm_k0.p, c->gm_v0.p, c->gm_k1.p, c->gm_v1.p, n, 32, c->gm_tmp.p, st);
  unsigned long long placed = 0;
  SG_CUDA(cudaMemcpyAsync(&placed, c->counters.p, sizeof(placed), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  if (placed)
    SG_CUDA(cudaMemcpyAsync(order, which ? c->gm_v1.p : c->gm_v0.p, sizeof(int32_t) * placed, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  *n_placed = (int64_t)placed;
  return 0;
}
