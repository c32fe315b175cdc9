// map_kernels.cuh -- per-pass mapping kernels (one reference sequence x one strand).
#pragma once

#include "common.cuh"

namespace sg {

// Scoring, as the kernels need it.
struct ScoreParams {
  int colour;
  int I;              // -i
  int Is;             // min(-i, 15): SIMD band half-width (main.c:302-313)
  int W;              // filter cells per hit: 2, 4, 8, 16 (run.c:64-101)
  int fm, fx, fo, fe; // filter scores: low bytes of |match|, |mismatch|, |open|, |extend|
  int fthr;           // filter threshold, min(z, 254) (alignment_simd.c:2525-2527)
  int pair[2][4];     // SCALE_SCORE(match|mismatch, level) (alignment.h:30, alignment.c:275-278)
  int gap_open, gap_ext;
  int min_score;      // -t
  // the packed nucleotide alignment (align_one_nuc): used when `packed`; its constants come
  // through the kernel parameters so that the multiply-adds stay multiply-adds
  int packed;
  uint32_t one;       // 1
  uint32_t open1;     // (gap_open << 13) + 1
  uint32_t open1_tc;  // open1 + (1 << 11) - (1 << 12): a corner-labelled cell as a top gap source
  uint32_t kt, kl;    // 4 (ext - open) - 2^22, 8 (ext - open) - 2^22 (modulo 2^32)
  uint32_t pw[32];    // 2^k
};

// filter width W for the SIMD half-width Is (run.c:64-101), and the scoring of a parameter set
int filter_width(int is);
ScoreParams make_score_params(const stormgpu_params& p);

struct ReadsDev {
  int64_t n;
  const uint8_t* codes;
  int64_t cstride;
  const uint8_t* levels;   // may be null
  int64_t lstride;
  const int16_t* lengths;
  // may be null; else the fused gather visits read order[k] k-th (reads grouped by length, so
  // that the candidate list, and with it the filter's and the alignment's blocks, is too)
  const int32_t* order;
};

struct IndexView {
  const int32_t* first[kMaxSeeds];
  const int32_t* map[kMaxSeeds];
};

struct PassBuffers {
  // filter -> flat list of passing candidates
  int32_t* pstart;      // per read: first slot
  int32_t* pcount;      // per read: number of passing candidates
  int32_t* p_read;      // per slot
  int32_t* p_diag;
  int64_t p_cap;
  unsigned long long* counters;  // [0] slots used, [1] overflow flag, [2] filter cells, [3] lookups, [4] positions
  // align outputs per slot
  int32_t* a_score;
  int32_t* a_bound;
  int16_t* a_pos;       // 4 per slot: best_i, best_j, best_i0, best_j0
  int32_t* a_tblen;
  uint8_t* a_tb;        // tbs bytes per slot (end-to-start order)
  int64_t tbs;
  uint32_t* a_scratch;  // direction bits, see align kernel
  int64_t scratch_words;
  // may be null; else a zeroed work cursor, and the align launch is a persistent grid of
  // align_workers() threads (scratch columns) taking slots from it
  unsigned long long* cursor;
  const int64_t* npass_dev;  // may be null; else the slot count is read from here
  int steal;                 // with a cursor: slots a warp takes at a time, a multiple of 32 (0 = 32)
  // Rounds (all null for one round over every slot).  The passing candidates of a read are
  // aligned in rounds of increasing rank (rank = slot - pstart[read]): round k takes the ranks
  // [align_round_bound(k), align_round_bound(k + 1)), listed in round_slots after the lists of
  // the rounds before it (round_count[k] slots); thr[read] holds the replay's running threshold
  // after the rounds before, below which a candidate can no longer be accepted, so that its
  // alignment may stop there.
  const int32_t* round_slots;
  const int64_t* round_count;  // [kMaxAlignRounds]
  int round;                   // the round of this launch
  int32_t* thr;                // per read; written by the replay of each round
  unsigned long long* cells;   // may be null; += band cells the alignment computed
};

constexpr int kMaxAlignRounds = 6;
// first rank of each round: 0, 8, 32, 128, 512, 2048, then every rank left
__host__ __device__ __forceinline__ int align_round_bound(int k, int rounds) {
  return k <= 0 ? 0 : k >= rounds ? 0x7fffffff : 8 << (2 * (k - 1));
}

void launch_reverse_reads(const ReadsDev& in, const uint8_t* first_levels, int colour,
                          uint8_t* rcodes, uint8_t* rlevels, cudaStream_t st);
void launch_init_results(int64_t n, stormgpu_hit* hits, uint8_t* mapped, uint8_t* tb, int64_t tbs,
                         cudaStream_t st);
void launch_align(const ReadsDev& r, const ScoreParams& sp, const uint8_t* genome,
                  const uint8_t* mask, int64_t slot0, int64_t nslots, PassBuffers& pb,
                  cudaStream_t st);
// scratch columns of a launch_align with a cursor (the threads of its persistent grid)
int64_t align_workers(int64_t nslots, const ScoreParams& sp);
void launch_replay(int64_t n, const ScoreParams& sp, int ref_id, int sense, PassBuffers& pb,
                   stormgpu_hit* hits, uint8_t* tb, int64_t tbs, uint8_t* mapped, cudaStream_t st);
// The slots of every round of a pass, in slot order within a warp's run: counts into
// round_count (zeroed by the caller), then the lists into round_slots.  `cursors` holds
// `rounds` zeroed counters.  With npass_dev (may be null) npass is an upper bound for the grid
// and the slot count is read from there.
void launch_round_lists(int64_t npass, const int64_t* npass_dev, int rounds, const int32_t* p_read,
                        const int32_t* pstart, int64_t* round_count, unsigned long long* cursors, int32_t* round_slots,
                        cudaStream_t st);
// Replay of round pb.round (the ranks of that round), continuing from pb.thr.
void launch_replay_round(int64_t n, const ScoreParams& sp, int ref_id, int sense, PassBuffers& pb, int rounds,
                         stormgpu_hit* hits, uint8_t* tb, int64_t tbs, uint8_t* mapped, cudaStream_t st);


}  // namespace sg
