// Whole-stream driver: splits the input into slabs of blocks, runs every
// stage on the GPU, and concatenates the slabs' parts of the .bz2 stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <mutex>
#include <vector>

namespace bz2g {

class Workspace;
namespace mlp {
struct SelectorTap;
}

// Block slots of every worker's workspace: the batched form packs up to this
// many short blocks into one slab.
constexpr int kBatchSlots = 1024;

struct StageTimes {
  // milliseconds of device time summed over slabs (CUDA events on each
  // worker's stream), filled when timing is enabled
  double rle1 = 0, bwt = 0, mtf = 0, rle2 = 0, huffman = 0, sizes = 0, place = 0;
  // totals over all blocks, for the HBM byte model
  // B = n + 10m + 28A + 14s + 5g + bits/8
  int64_t blocks = 0, n = 0, m = 0, A = 0, s = 0, g = 0, bits = 0;
  // radix scatter launches (when timing is enabled): count, summed device
  // ms, and algorithmic bytes (each element's item read and written once)
  int64_t scatter_launches = 0;
  double scatter_ms = 0, scatter_bytes = 0;
  // BWT rounds (when timing is enabled), summed over slabs by round index:
  // r = 0 the first sort (standing for the oracle's rounds h = 1, 2), r >= 1
  // the doubling round with shift 4 * 2^(r-1).  round_active: rotations the
  // byte model charges to the round; round_ms: device time.
  double round_ms[24] = {};
  int64_t round_active[24] = {};
  // blocks whose tables came from the learned selector, and blocks with six
  // tables (the learned selector's domain; the rest fell back to plain)
  int64_t learned_blocks = 0, six_table_blocks = 0;
};

struct CompressorConfig {
  int slab_blocks = 384;
  int workers = 4;
  int64_t max_block_bytes = 900000;
  bool time_stages = false;
  // Learned table selector: packed weights on this engine's device
  // (selector.h), or nullptr for the reference's plain selector.
  const uint8_t *selector = nullptr;
  // Selection passes of the plain selector (the reference's 4; 1 is the
  // single-pass baseline the learned form is measured against).
  int plain_passes = 4;
  // Training-set tap: every block with six tables appends its groups and the
  // plain selector's choices (deterministic order with one worker).
  const mlp::SelectorTap *tap = nullptr;
  // Block format of compress / compress_device.  Reference: runs cut at 259
  // and blocks of at most max_block_bytes raw bytes.  bzip2 1.0.8: runs cut
  // at 255 and blocks of any raw length whose RLE1 output is at most m_cap
  // bytes (the bzip2 split; slabs take fewer blocks when they are long).
  int run_cut = 259;
  int64_t m_cap = 0;
};

// Destination of a stream: a malloc'd buffer that this library grows (and
// the caller may take over and free()), or a caller buffer of fixed capacity.
struct ByteSink {
  uint8_t *data = nullptr;
  size_t size = 0, cap = 0;
  bool owned = true;
  bool pinned = false;  // data is page-locked: device copies land in it directly
  bool device = false;  // data is device memory (caller buffer)
  ByteSink() = default;
  ByteSink(uint8_t *p, size_t c);  // caller buffer
  ~ByteSink();
  ByteSink(const ByteSink &) = delete;
  ByteSink &operator=(const ByteSink &) = delete;
  void reserve(size_t c);          // owned only
  uint8_t *release();              // hand the owned buffer to the caller
};

class Compressor {
 public:
  explicit Compressor(const CompressorConfig &cfg);
  ~Compressor();
  // Compress the blocks (host memory; pinned memory makes the copies
  // asynchronous) into one stream with header digit `level`, written at
  // out.size onward.
  void compress(const uint8_t *const *ptrs, const int *lens, int nblocks, int level,
                ByteSink &out, StageTimes *times = nullptr);
  // Same, with the blocks already in device memory (raw bytes of block b at
  // d_ptrs[b]).
  void compress_device(const uint8_t *const *d_ptrs, const int *lens, int nblocks, int level,
                       ByteSink &out, StageTimes *times = nullptr);
  // A part of a stream for sharding one stream over several GPUs: the blocks'
  // bits from bit 0 of out (device memory, caller buffer), no stream header
  // and no end-of-stream marker.  *bits: the part's bit count; *crc_fold: the
  // blocks' CRCs folded as the stream CRC is (rotate left 1, xor) from 0.
  void compress_part(const uint8_t *const *ptrs, const int *lens, int nblocks, bool on_device,
                     ByteSink &out, int64_t *bits, uint32_t *crc_fold,
                     StageTimes *times = nullptr);
  // Convenience for callers holding a std::vector (appends).
  void compress(const uint8_t *const *ptrs, const int *lens, int nblocks, int level,
                std::vector<uint8_t> &out, StageTimes *times = nullptr);
  // Batched form: every item becomes its own stream (header digit
  // item.level, blocks of item.block_bytes raw bytes); all blocks of all
  // items run through shared slabs in order of decreasing length, and the
  // streams are written back to back into out (offsets: count + 1 entries).
  // Each stream equals compress() of that item alone.
  struct Item {
    const uint8_t *ptr;
    int64_t n;
    int level;
    int block_bytes;
  };
  void compress_batch(const Item *items, int count, bool on_device, ByteSink &out,
                      std::vector<size_t> &offsets, StageTimes *times = nullptr);
  // Batched form tuning, by block length: a slab whose longest block has at
  // most max_len raw bytes takes up to slab_blocks blocks (within the
  // workspace's capacities), and a call runs on up to `workers` worker
  // streams (chosen by its byte-weighted median block length).  Entries are
  // kept sorted by max_len; an empty table keeps config().slab_blocks blocks
  // per slab and every worker.
  struct BatchTune {
    int max_len, slab_blocks, workers;
  };
  void set_batch_tuning(const std::vector<BatchTune> &table);
  const CompressorConfig &config() const { return cfg_; }
  int device() const { return device_; }

 private:
  struct Worker;
  void run(const uint8_t *const *ptrs, const int *lens, int nblocks, int level, bool on_device,
           ByteSink &out, StageTimes *times, bool part = false, int64_t *part_bits = nullptr,
           uint32_t *part_crc = nullptr);
  uint32_t *arena_take(int64_t words, size_t *chunk, int64_t *used, int64_t *base);
  BatchTune tune_for(int len) const;
  void reserve(int blocks);
  static constexpr int64_t kArenaChunkWords = int64_t(1) << 28;  // 1 GiB
  CompressorConfig cfg_;
  int device_ = 0;
  std::vector<std::unique_ptr<Worker>> workers_;
  int slab_capacity_ = 0;                      // blocks the workers' workspaces hold
  std::mutex call_mu_;                         // one call at a time per engine
  std::vector<BatchTune> tune_;               // batched form: slab shapes by block length
  std::vector<uint32_t *> arena_chunks_;       // batched form: block bits
  std::vector<int64_t> arena_chunk_words_;
  uint32_t *splice_out_ = nullptr;             // batched form: spliced streams
  int64_t splice_out_words_ = 0;
  int64_t *splice_meta_ = nullptr;             // per block: source, destination bit, bits
  int64_t splice_meta_blocks_ = 0;
};

// Upper bound of the stream size for n bytes in nblocks blocks.
size_t stream_bound(int64_t n, int64_t nblocks);

// End-of-stream marker and combined CRC at stream bit `bit` of out (host),
// counted from out.data + base; grows out.size to the padded end.
void put_eos(ByteSink &out, size_t base, int64_t bit, uint32_t crc);

}  // namespace bz2g
