// bzip2 1.0.8's block split on the GPU (split.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace bz2g {

// Block ends (raw offsets, ascending, the last one n) of bzip2 1.0.8's split
// of the n device bytes at d_in at `level` (blocks of at most
// 100000 * level - 19 RLE1 bytes before their last run, runs cut at 255).
std::vector<int64_t> bzip2_split(const uint8_t *d_in, int64_t n, int level, cudaStream_t st);
// Upper bound of the number of blocks of that split.
int64_t bzip2_split_max_blocks(int64_t n, int level);

}  // namespace bz2g
