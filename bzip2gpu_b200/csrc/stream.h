// Streaming compression with bounded host memory.
//
// The reference reads its whole input into one pinned buffer per 900,000-byte
// chunk (src/utils/io.cpp:16, one cudaMallocHost each) and writes the
// container after every block is done (src/compression/compress.cu:284-375).
// Here blocks arrive in order in groups; each group is compressed on the GPU
// into a part (Compressor::compress_part), the part is spliced on the device at
// the stream's running bit phase, and its finished bytes go to a sink while
// the next group is read.  Host memory: the input ring and one group.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>

#include "compressor.h"

namespace bz2g {

class StreamWriter {
 public:
  using Sink = std::function<void(const uint8_t *, size_t)>;
  StreamWriter(Compressor &c, int level, Sink sink);
  ~StreamWriter();
  StreamWriter(const StreamWriter &) = delete;
  StreamWriter &operator=(const StreamWriter &) = delete;

  // Compress the blocks (host or device memory) and emit the finished bytes.
  void add(const uint8_t *const *ptrs, const int *lens, int nblocks, bool on_device);
  // End-of-stream marker and combined CRC; emits the rest of the stream.
  void finish();
  int64_t bytes_out() const { return bytes_out_; }

 private:
  void emit(const uint8_t *p, size_t n);
  Compressor &c_;
  int level_;
  Sink sink_;
  bool header_done_ = false;
  uint8_t pending_ = 0;   // the stream's last, partial byte (top pending_bits_ bits)
  int pending_bits_ = 0;
  uint32_t crc_ = 0;
  int64_t bytes_out_ = 0;
  uint8_t *d_part_ = nullptr;
  size_t part_cap_ = 0;
  uint32_t *d_stage_ = nullptr;
  size_t stage_words_ = 0;
  int64_t *d_meta_ = nullptr;
  size_t meta_cap_ = 0;
  uint8_t *h_stage_ = nullptr;  // pinned
  size_t h_stage_cap_ = 0;
};

// The engine the whole-stream C-ABI calls use on this device (blocks of up to
// max_block_bytes).
Compressor &default_engine(int64_t max_block_bytes);

}  // namespace bz2g

struct BZFileInputStream;

namespace bz2g {

// Blocks per GPU group of the streaming path: enough for every worker of the
// default engine to have slabs in flight.
constexpr int kGroupBlocks = 384;

// Feeds every chunk of `in` through `w` in groups of up to group_blocks
// blocks (pooled chunks, given back after each group), then finishes the
// stream.
void compress_input_stream(BZFileInputStream &in, StreamWriter &w,
                           int group_blocks = kGroupBlocks);

}  // namespace bz2g
