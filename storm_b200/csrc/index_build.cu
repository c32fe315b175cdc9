// index_build.cu -- device-resident spaced-seed index of one reference sequence for one seed:
// a CSR table first[4^w + 1] (offsets) / map[] (positions, ascending per key), the layout of
// the reference's contiguous index (index.c:161-188, read by index__get_extern_next_hit,
// index.c:212-241).
//
// Build = seed keys of every indexed position (kernel) -> stable LSD radix sort of (key, pos)
// -> per-key runs of the sorted list (start, count) -> repeat filter (exact integer moments;
// the host turns them into the largest admissible count) -> a scan of the kept counts ->
// compaction into the CSR.  HBM-streaming work.
#include <cmath>
#include <vector>

#include "index_build.cuh"
#include "radix.cuh"

namespace sg {

// Indexed positions come as intervals [a, b); t-th indexed position = a_k + (t - before_k).
__global__ void seed_keys_kernel(const uint8_t* __restrict__ codes, const int64_t* __restrict__ ia,
                                 const int64_t* __restrict__ ibefore, int nint, int64_t total,
                                 SeedDev seed, uint32_t* __restrict__ keys, uint32_t* __restrict__ pos) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  int lo = 0, hi = nint - 1;
  while (lo < hi) {  // last interval with before <= t
    int mid = (lo + hi + 1) >> 1;
    if (ibefore[mid] <= t) lo = mid; else hi = mid - 1;
  }
  int64_t p = ia[lo] + (t - ibefore[lo]);
  uint32_t key = 0;
  for (int c = 0; c < seed.n_care; ++c) key = (key << 2) | (uint32_t)code_at(codes, p + seed.care[c]);
  keys[t] = key;
  pos[t] = (uint32_t)p;
}

// Runs of equal keys in the sorted list: start[k] = first index of key k, end[k] = one past its
// last (both left at 0 for absent keys), so that count = end - start with no atomics.
__global__ void key_runs_kernel(const uint32_t* __restrict__ skeys, int64_t n, int32_t* __restrict__ start,
                                int32_t* __restrict__ end) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t k = skeys[t];
  if (t == 0 || skeys[t - 1] != k) start[k] = (int32_t)t;
  if (t == n - 1 || skeys[t + 1] != k) end[k] = (int32_t)(t + 1);
}

__global__ void run_counts_kernel(const int32_t* __restrict__ start, int64_t nkeys, int32_t* __restrict__ counts) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nkeys) counts[k] -= start[k];
}

__global__ void moments_kernel(const int32_t* __restrict__ counts, int64_t nkeys,
                               unsigned long long* __restrict__ out) {
  unsigned long long s2 = 0, nocc = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nkeys; k += (int64_t)gridDim.x * blockDim.x) {
    long long c = counts[k];
    if (c > 0) { s2 += (unsigned long long)(c * c); nocc++; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    nocc += __shfl_xor_sync(0xffffffffu, nocc, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], s2);
    atomicAdd(&out[1], nocc);
  }
}

__global__ void kept_kernel(const int32_t* __restrict__ counts, int64_t nkeys, int32_t cmax,
                            int32_t* __restrict__ kept) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nkeys) {
    int32_t c = counts[k];
    kept[k] = c <= cmax ? c : 0;
  }
}

__global__ void csr_fill_kernel(const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ spos,
                                int64_t n, const int32_t* __restrict__ counts,
                                const int32_t* __restrict__ allstart, const int32_t* __restrict__ first,
                                int32_t cmax, int32_t* __restrict__ map) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t k = skeys[t];
  if (counts[k] <= cmax) map[first[k] + (t - allstart[k])] = (int32_t)spos[t];
}

// Host simulation of the position loop of index.c:65-96 at interval granularity: windows are
// skipped while i + span >= start of the next masked region, i jumps to end-1 of that region
// (re-checking the following regions), and that position is indexed without re-testing the
// loop bound.  Returns the intervals of indexed positions, in increasing order.
void indexed_intervals(int64_t n_codes, int span, const int32_t* rs, const int32_t* re, int nreg,
                       std::vector<int64_t>& a, std::vector<int64_t>& b) {
  a.clear();
  b.clear();
  int64_t map_size = n_codes - span + 1;
  if (map_size <= 0 || span >= n_codes) return;
  int64_t i = 0;
  int r = 0;
  while (i < map_size) {
    int64_t trig = (r < nreg) ? std::max<int64_t>(i, (int64_t)rs[r] - span) : map_size;
    if (trig >= map_size) {
      a.push_back(i); b.push_back(map_size);
      break;
    }
    if (trig > i) { a.push_back(i); b.push_back(trig); }
    i = trig;
    while (r < nreg && i + span >= rs[r]) { i = (int64_t)re[r] - 1; r++; }
    if (!a.empty() && b.back() == i) b.back() = i + 1;
    else { a.push_back(i); b.push_back(i + 1); }
    i++;
  }
}

// Largest count c that the repeat filter keeps: c is erased iff c - avg > l * sd with
// avg = sum(c^2)/N^2 and sd^2 = sum_{c>0}(c - avg)^2 / N (index.c:117-155), both from the exact
// integer moments, compared in long double.
int32_t repeat_cutoff(int stdev_distance, int64_t N, unsigned long long s2, unsigned long long nocc) {
  if (stdev_distance <= 0 || N <= 0) return INT32_MAX;
  long double n = (long double)N;
  long double avg = (long double)s2 / n / n;
  long double var = ((long double)s2 - 2.0L * avg * n + (long double)nocc * avg * avg) / n;
  long double sd = sqrtl(var > 0 ? var : 0);
  auto erased = [&](long double c) { return (c - avg) > (long double)stdev_distance * sd; };
  long double guess = floorl(avg + (long double)stdev_distance * sd);
  if (guess > (long double)INT32_MAX) return INT32_MAX;
  if (guess < 0) guess = 0;
  int64_t c = (int64_t)guess;
  while (c + 1 <= INT32_MAX && !erased((long double)(c + 1))) c++;
  while (c > 0 && erased((long double)c)) c--;
  return (int32_t)c;
}

int build_one_index(const uint8_t* d_codes, int64_t n_codes, const int32_t* rs, const int32_t* re,
                    int nreg, const SeedDev& seed, int stdev_distance, DevIndex* out,
                    cudaStream_t st, int64_t* launches) {
  std::vector<int64_t> a, b;
  indexed_intervals(n_codes, seed.span, rs, re, nreg, a, b);
  const int64_t nkeys = (int64_t)1 << (2 * seed.weight);
  out->weight = seed.weight;
  out->nkeys = nkeys;
  std::vector<int64_t> before(a.size());
  int64_t total = 0;
  for (size_t k = 0; k < a.size(); ++k) { before[k] = total; total += b[k] - a[k]; }
  SG_CUDA(cudaMallocAsync(&out->first, sizeof(int32_t) * (nkeys + 1), st));
  SG_CUDA(cudaMemsetAsync(out->first, 0, sizeof(int32_t) * (nkeys + 1), st));
  out->map = nullptr;
  out->n = 0;
  if (total == 0) return 0;
  if (total > INT32_MAX) { sg_set_error("sequence too long for 32-bit positions"); return STORMGPU_EINVAL; }
  int64_t* d_iv;
  uint32_t *k0, *v0, *k1, *v1;
  int32_t *counts, *kept, *allstart;
  unsigned long long* mom;
  void* tmp;
  const int64_t tmpb = std::max<int64_t>(radix_tmp_bytes(total), (scan_tmp_elems(nkeys + 1) + 8) * 4);
  SG_CUDA(cudaMallocAsync(&d_iv, sizeof(int64_t) * 2 * a.size(), st));
  SG_CUDA(cudaMallocAsync(&k0, sizeof(uint32_t) * total, st));
  SG_CUDA(cudaMallocAsync(&v0, sizeof(uint32_t) * total, st));
  SG_CUDA(cudaMallocAsync(&k1, sizeof(uint32_t) * total, st));
  SG_CUDA(cudaMallocAsync(&v1, sizeof(uint32_t) * total, st));
  SG_CUDA(cudaMallocAsync(&counts, sizeof(int32_t) * nkeys, st));
  SG_CUDA(cudaMallocAsync(&kept, sizeof(int32_t) * (nkeys + 1), st));
  SG_CUDA(cudaMallocAsync(&allstart, sizeof(int32_t) * (nkeys + 1), st));
  SG_CUDA(cudaMallocAsync(&mom, sizeof(unsigned long long) * 2, st));
  SG_CUDA(cudaMallocAsync(&tmp, tmpb, st));
  SG_CUDA(cudaMemcpyAsync(d_iv, a.data(), sizeof(int64_t) * a.size(), cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemcpyAsync(d_iv + a.size(), before.data(), sizeof(int64_t) * a.size(), cudaMemcpyHostToDevice, st));
  int64_t L = 0;
  const int TB = 256;
  seed_keys_kernel<<<(unsigned)((total + TB - 1) / TB), TB, 0, st>>>(d_codes, d_iv, d_iv + a.size(),
                                                                       (int)a.size(), total, seed, k0, v0);
  L++;
  int which = radix_sort_pairs(k0, v0, k1, v1, total, 2 * seed.weight, tmp, st);
  L += 3 * ((2 * seed.weight + kRadixBits - 1) / kRadixBits);
  uint32_t* sk = which ? k1 : k0;
  uint32_t* sv = which ? v1 : v0;
  SG_CUDA(cudaMemsetAsync(counts, 0, sizeof(int32_t) * nkeys, st));
  SG_CUDA(cudaMemsetAsync(allstart, 0, sizeof(int32_t) * nkeys, st));
  key_runs_kernel<<<(unsigned)((total + TB - 1) / TB), TB, 0, st>>>(sk, total, allstart, counts);
  run_counts_kernel<<<(unsigned)((nkeys + TB - 1) / TB), TB, 0, st>>>(allstart, nkeys, counts);
  SG_CUDA(cudaMemsetAsync(mom, 0, sizeof(unsigned long long) * 2, st));
  moments_kernel<<<592, TB, 0, st>>>(counts, nkeys, mom);
  L += 3;
  unsigned long long hm[2];
  SG_CUDA(cudaMemcpyAsync(hm, mom, sizeof(hm), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  int32_t cmax = repeat_cutoff(stdev_distance, total, hm[0], hm[1]);
  kept_kernel<<<(unsigned)((nkeys + TB - 1) / TB), TB, 0, st>>>(counts, nkeys, cmax, kept);
  exclusive_scan<int32_t, int32_t>(kept, out->first, nkeys, out->first + nkeys, (int32_t*)tmp, st);
  L += 1 + 3;
  int32_t nmap = 0;
  SG_CUDA(cudaMemcpyAsync(&nmap, out->first + nkeys, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  out->n = nmap;
  SG_CUDA(cudaMallocAsync(&out->map, sizeof(int32_t) * std::max<int64_t>(nmap, 1), st));
  csr_fill_kernel<<<(unsigned)((total + TB - 1) / TB), TB, 0, st>>>(sk, sv, total, counts, allstart,
                                                                      out->first, cmax, out->map);
  L++;
  SG_CUDA(cudaGetLastError());
  cudaFreeAsync(d_iv, st); cudaFreeAsync(k0, st); cudaFreeAsync(v0, st); cudaFreeAsync(k1, st);
  cudaFreeAsync(v1, st); cudaFreeAsync(counts, st); cudaFreeAsync(kept, st);
  cudaFreeAsync(allstart, st); cudaFreeAsync(mom, st); cudaFreeAsync(tmp, st);
  if (launches) *launches += L;
  out->positions_indexed = total;
  out->cmax = cmax;
  return 0;
}

}  // namespace sg
