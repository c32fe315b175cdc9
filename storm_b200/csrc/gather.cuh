// gather.cuh -- fused hit gather (gather.cu).
#pragma once

#include "map_kernels.cuh"

namespace sg {

struct GatherOut {
  int32_t* fr;                   // flat list: read of each candidate
  int32_t* fd;                   // flat list: diagonal of each candidate
  int64_t cap;                   // capacity of fr / fd
  unsigned long long* counters;  // [3] key lookups, [4] index positions, [7] flat cursor, [8] overflow
  // reads with more positions than a warp holds, with their position counts: up to
  // kSmallGatherCap in (small_list, small_h), more in (big_list, big_h); counts [0] big, [2] small
  int32_t* big_list;
  int32_t* big_h;
  int32_t* small_list;
  int32_t* small_h;
  int32_t* big_count;
  unsigned long long* cursor;    // zeroed work cursor of the fused gather (reads taken so far)
  int reads_per_steal;           // reads a warp takes from the cursor at a time (>= 1)
  int warp_cap;                  // index positions a warp holds in shared memory, <= kMaxWarpCap;
                                 // reads with more go to the block kernel
};

constexpr int kMaxWarpCap = 1536;

constexpr int kBlockGatherCap = 65536;

// The seed family travels with every launch (a kernel parameter), so that mapping calls with
// different seed families can run concurrently on different streams.
void launch_gather_fused(const ReadsDev& rd, const IndexView& ix, int I, const GatherOut& go, const SeedSet& seeds,
                         cudaStream_t st);
// The nlist reads of `list` with their position counts `list_h` (with nlist_dev, which may be
// null, the count is read from there when the kernel starts and nlist is only nonzero), a
// persistent grid of `grid` blocks (at most gather_block_grid(smem) useful) taking reads from the
// zeroed `cursor`; scratch holds 2 * cap words per block.  Reads with more than `cap` positions
// are appended to (huge_list, huge_h), counted in huge_count.  smem: the slices in shared memory,
// for lists whose reads have at most kSmallGatherCap positions.
constexpr int kSmallGatherCap = 4096;
void launch_gather_block(const ReadsDev& rd, const IndexView& ix, int I, const int32_t* list, const int32_t* list_h,
                         int64_t nlist, const int32_t* nlist_dev, const GatherOut& go, int32_t* scratch, int cap,
                         int64_t grid, unsigned long long* cursor, int32_t* huge_list, int32_t* huge_h,
                         int32_t* huge_count, bool smem, const SeedSet& seeds, cudaStream_t st);
int64_t gather_block_grid(bool smem);

}  // namespace sg
