// Slab engine: every stage runs over a batch ("slab") of independent blocks.
//
// HBM layout of a slab (all per-block arrays are indexed by one shared
// element layout, so a kernel finds a block's data at off[b]):
//   raw      uint8   block b at raw_off[b] (16-byte aligned), raw_len[b] bytes
//   rle1     uint8   block b at off[b], m[b] bytes           (off[b] % kTile == 0)
//   sa, isa, kpos[2] int32 at off[b], m[b] entries (block-local indices)
//   keys[2]  uint64, vals[2] uint32: radix sort ping-pong, same layout
//   last     uint8   BWT last column, same layout
//   mtf      uint8   same layout
//   rle2     uint16  same layout, s[b] <= m[b] + 1 <= cap[b] symbols
//   sel      uint8   selectors at off[b]/32 (cap[b]/32 >= cap[b]/50 + 1)
//   out      uint32  big-endian words of the slab's part of the .bz2 stream
// Tiles of kTile elements never cross blocks; tile_block[t] names the owner.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"

namespace bz2g {

// Per-slab plan, built on the host from the raw block lengths.
// Workspace a block of L raw bytes takes in a slab.  m_cap > 0 bounds its
// RLE1 bytes (the bzip2 split's blocks: many raw bytes, bounded RLE1 output).
struct BlockNeeds {
  int64_t raw, elems;
  int raw_tiles, tiles, group_tiles;
};
BlockNeeds block_needs(int64_t L, int64_t m_cap);

struct SlabPlan {
  int nblocks = 0;
  // RLE1 run cut: 259 (the reference: 4 + 255) or 255 (bzip2 1.0.8)
  int run_cut = 259;
  int64_t m_cap = 0;
  std::vector<int64_t> raw_off, off, cap;
  std::vector<int> raw_len;
  std::vector<int> rt_block, rt_start, rt_first;  // raw tiles (rt_first: nblocks+1)
  std::vector<int> tile_block;          // element tiles
  std::vector<int> gt_block, gt_first;  // group tiles (kGroupTile groups each)
  std::vector<int> gt_begin;            // first group tile of each block (nblocks+1)
  int64_t raw_total = 0, elem_total = 0;
  int max_m_bound = 0;
  void build(const int *lens, int n, int run_cut = 259, int64_t m_cap = 0);
};

constexpr int kGroupTile = 128;  // 50-symbol groups per group tile
constexpr int kMaxRadix = 512;   // widest radix sort digit (9 bits)

// Device pointers of one slab, passed to kernels by value.
struct SlabDev {
  int nblocks, ntiles, n_raw_tiles, n_group_tiles;
  int run_cut;  // RLE1 run cut (259 or 255)
  // plan
  const int64_t *raw_off, *off, *cap;
  const int *raw_len, *rt_block, *rt_start, *rt_first, *tile_block, *gt_block, *gt_first, *gt_begin;
  // data
  uint8_t *raw, *rle1, *last, *mtf;
  int32_t *sa, *isa;
  int32_t *kpos[2];                    // BWT: sorted-array position of each active rotation
  uint64_t *keys[2];
  uint32_t *vals[2];
  uint16_t *rle2;
  uint8_t *sel, *sel_mtf;
  uint32_t *out;
  // per-tile scratch
  int32_t *tile_a, *tile_b, *tile_c, *tile_d;  // [ntiles] or [n_raw_tiles]
  uint32_t *tile_hist;                 // [ntiles * kMaxRadix]: radix sort tile digit counts
  uint32_t *sort_base;                 // [nblocks * kMaxRadix]: radix sort digit bases
  int32_t *blk_count;                  // [nblocks]: radix sort tiles counted (reset by the last)
  int32_t *tile_last;                  // [ntiles * 256]
  uint32_t *gt_bits;                   // [n_group_tiles]
  uint32_t *grp_bits;                  // per group, at sel layout
  // per-block
  int32_t *m, *s, *n_in_use, *orig_ptr, *n_groups, *n_sel;
  uint32_t *crc, *crc_acc, *present;  // present: 8 words per block
  int32_t *freq;                       // [nblocks * 258]
  uint8_t *len;                        // [nblocks * 6 * 258]
  int32_t *code;                       // [nblocks * 6 * 258]
  int32_t *rfreq;                      // [nblocks * 6 * 258]
  int32_t *learned;                    // [nblocks]: table selection by the learned selector
  int32_t *rfreq_m;                    // [nblocks * 6 * 258]: the MLP's per-table counts
  uint8_t *len2;                       // [nblocks * 6 * 258]: learned form, the plain
                                       // selector's tables of learned blocks
  uint8_t *sel2;                       // learned form: the plain selector's second-pass
                                       // selectors of learned blocks (sel layout)
  int32_t *rfreq2;                     // [nblocks * 6 * 258]: their per-table counts
  int32_t *plain_left;                 // [nblocks]: plain passes still to run (learned form)
  int32_t *err;                        // device error word of the tensor-core kernels
  int32_t *sort_len, *done, *ngroups;  // BWT control (ngroups: groups among active rotations)
  int32_t *act_len;                    // BWT: active rotations entering the next round
  int32_t *tile_list;                  // BWT: tiles holding active rotations [ntiles]
  // The tiles that hold data, listed in block order (a block's workspace is
  // sized for its worst-case RLE1 output, so most of its tiles can be empty):
  // element tiles of the m[b] RLE1 bytes, and group tiles of the
  // ceil(s[b] / 50) groups.  live (pinned host) [0], [1]: their counts once
  // known for this slab, -1 before (kernels then run over every tile); [2]:
  // the slab's largest m, known with [0]; [4..6]: staging.
  int32_t *vt_list, *vg_list;
  int *live;
  int32_t *warp_last, *warp_act;       // BWT: per 512-element warp span [ntiles * 8]: last
                                       // head, then its carry; active count, then offset
  int64_t *active_sum;                 // A: rotations in non-singleton groups, summed over rounds
  int32_t *pstat;                      // [nblocks * 8]: heads and singletons at prefix 1,2,4,8
  int64_t *hdr_bits, *pay_bits, *blk_start;
  // radix sort control
  int32_t *sort_ctl;                   // [0]=cur key buffer, [1]=nontrivial flag,
                                       // [2]=blocks still sorting, [3]=cur kpos buffer,
                                       // [4]=tiles of the next round, [5]=tile list fill,
                                       // [6]=rotations entering the next round,
                                       // [8..9]=u64 rotations the first sort's model charges
                                       // [10], [11]=tile-list counts, [12]=largest m
  int32_t *h_flags;                    // pinned host mirror of small counters
  // stream state: [0] = bit offset (u64), [1] = stream crc, [2] = slab first word,
  // [3] = slab word count
  uint64_t *stream;
  // optional per-launch timing of the radix scatter (host-side fields, only
  // read on the host): events around each launch, the elements each launch
  // moved (device counters) and its bytes per element
  int kt_on;
  cudaEvent_t *kt_ev;       // [2 * kMaxTimedLaunches]
  int *kt_n;                // launches recorded in this slab
  int *kt_bpe;              // [kMaxTimedLaunches]
  uint64_t *kt_elems;       // device [kMaxTimedLaunches]
  // optional per-round timing of the BWT (host-side fields, with kt_on):
  // events around round r (r = 0: the first sort and its ranking; r >= 1:
  // the doubling round with shift 4 * 2^(r-1)), rounds recorded, and the
  // rotations the round's model charges (r = 0: those the first sort stands
  // for, the oracle's rounds h = 1 and 2; r >= 1: active rotations entering
  // the round)
  cudaEvent_t *rt_ev;       // [2 * kMaxRounds]
  int *rt_n;
  int64_t *rt_act;          // [kMaxRounds]
};

constexpr int kMaxTimedLaunches = 96;
constexpr int kMaxRounds = 24;

// Owns the device buffers of a slab context (sized for a maximum slab).
class Workspace {
 public:
  Workspace(int max_blocks, int64_t max_raw, int64_t max_elems, int max_tiles,
            int max_raw_tiles, int max_group_tiles);
  ~Workspace();
  // Sized for slabs of up to max_blocks blocks of up to max_block_bytes each;
  // per-block arrays for max(max_blocks, block_slots) blocks, so a slab of
  // shorter blocks can hold more of them (within the same element, raw-byte
  // and tile capacities).
  static Workspace *create_for(int max_blocks, int64_t max_block_bytes, int block_slots = 0);
  Workspace(const Workspace &) = delete;
  Workspace &operator=(const Workspace &) = delete;

  // Upload a plan (async on `st`; the plan's host vectors must stay alive until
  // the stream reaches this point, so they are copied into pinned staging).
  void upload_plan(const SlabPlan &p, cudaStream_t st);
  SlabDev dev;
  int max_blocks;
  int64_t max_raw, max_elems, out_words;
  int max_tiles, max_raw_tiles, max_group_tiles;
  void *pinned_plan = nullptr;
  size_t pinned_plan_bytes = 0;

 private:
  std::vector<void *> allocs_;
  void *plan_dev_ = nullptr;
  void *alloc(size_t bytes);
};

// The listed tiles of the slab (built on the first call after m, or s, is
// final; the count is read back, one synchronisation of `st`): the element
// tiles holding RLE1 bytes, and the group tiles holding 50-symbol groups.
// Return -1 when the slab has no list (launch over every tile then).
int live_tiles(const SlabDev &d, cudaStream_t st);
int live_group_tiles(const SlabDev &d, cudaStream_t st);

// ------------------------------------------------------------------ stages
void stage_rle1_crc(const SlabDev &d, cudaStream_t st);
// BWT over rle1[off[b], m[b]) -> sa.  max_m: host bound of max m[b].
void stage_bwt(const SlabDev &d, int max_m, cudaStream_t st);
void stage_mtf(const SlabDev &d, cudaStream_t st);
void stage_rle2(const SlabDev &d, cudaStream_t st);
// Table selection, code lengths and codes.  learned: packed selector weights
// (selector.h) for the learned form, or nullptr for the reference's plain
// selector.  plain_passes: selection passes of the plain selector (the
// reference runs 4; 1 gives the single-pass baseline of the learned form's
// measurements).  mlp_sel_out (optional): a copy of the selector array right
// after the MLP's assignment (mlp_sel_bytes from d.sel), for tests.
void stage_huffman(const SlabDev &d, cudaStream_t st, const uint8_t *learned = nullptr,
                   int plain_passes = kIters, uint8_t *mlp_sel_out = nullptr,
                   size_t mlp_sel_bytes = 0);
// payload bit counts, header bit counts and selector MTF
void stage_sizes(const SlabDev &d, cudaStream_t st);
// payload bit counts only (tables, selectors and symbols already in place)
void stage_sizes_payload_only(const SlabDev &d, cudaStream_t st);
// Zero the slab's output words and write headers and payloads at their final
// stream positions.  slab_start_bit: stream bit offset of the slab's first
// block; w0: stream word index of out[0]; nwords: words to zero.
void stage_place(const SlabDev &d, int64_t slab_start_bit, int64_t w0, int64_t nwords,
                 cudaStream_t st);

// Kernel launches issued by this library so far.
int64_t launch_count();

// Batched form: blocks placed word-aligned in an arena (d.blk_start filled by
// the caller), then spliced to their bit positions in the output streams.
void stage_place_arena(const SlabDev &d, uint32_t *arena, int64_t w0, int64_t nwords,
                       cudaStream_t st);
// src_addr: device address of each block's first word.
void launch_splice(const int64_t *src_addr, const int64_t *dst_bit, const int64_t *nbits,
                   int nblocks, uint32_t *out, cudaStream_t st);

// Individual pieces used by the per-stage C-ABI.
void launch_crc_only(const SlabDev &d, cudaStream_t st);
void launch_pack_words(const SlabDev &d, uint32_t *words, cudaStream_t st);

}  // namespace bz2g
