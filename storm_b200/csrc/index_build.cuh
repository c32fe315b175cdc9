// index_build.cuh -- CSR seed index on the device (see index_build.cu).
#pragma once

#include <vector>

#include "common.cuh"

namespace sg {

struct DevIndex {
  int weight = 0;
  int64_t nkeys = 0;            // 4^weight
  int32_t* first = nullptr;     // nkeys + 1 offsets
  int32_t* map = nullptr;       // first[nkeys] positions
  int64_t n = 0;                // first[nkeys]
  int64_t positions_indexed = 0;
  int32_t cmax = 0;             // largest count kept by the repeat filter
};

void indexed_intervals(int64_t n_codes, int span, const int32_t* rs, const int32_t* re, int nreg,
                       std::vector<int64_t>& a, std::vector<int64_t>& b);
int32_t repeat_cutoff(int stdev_distance, int64_t N, unsigned long long s2, unsigned long long nocc);
int build_one_index(const uint8_t* d_codes, int64_t n_codes, const int32_t* rs, const int32_t* re,
                    int nreg, const SeedDev& seed, int stdev_distance, DevIndex* out,
                    cudaStream_t st, int64_t* launches);

}  // namespace sg
