// Whole-stream driver (reference: src/compression/compress.cu:184-378).
//
// The reference compresses one block per host thread and stream, then writes
// the container serially on the host.  Here each worker owns a slab workspace
// and a stream and runs every stage for a whole slab of blocks on the GPU;
// the only serial host work per slab is a prefix over its blocks' bit sizes
// (for the stream position and the combined CRC) and appending its bytes.
// Slabs finish in any order; offsets and appends are taken in slab order.
#include "compressor.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <exception>
#include <mutex>
#include <thread>

#include "engine.h"
#include "selector.h"

namespace bz2g {

static_assert(kMaxRounds == sizeof(StageTimes::round_ms) / sizeof(double),
              "per-round statistics size");

struct Compressor::Worker {
  Workspace *ws = nullptr;
  cudaStream_t st = nullptr;
  uint8_t *h_out = nullptr;
  size_t h_out_cap = 0;
  int64_t *h_sizes = nullptr;  // [2 * max_blocks] hdr, pay
  int32_t *h_cnt = nullptr;    // [5 * max_blocks] m, s, n_sel, learned, n_groups
  int64_t *h_act = nullptr;    // [max_blocks] A
  uint32_t *h_crc = nullptr;
  int32_t *h_err = nullptr;    // the workspace's device error word
  int slots = 0;               // blocks a slab may hold (stride of the host arrays)
  cudaEvent_t ev[8] = {};
  cudaEvent_t kt_ev[2 * kMaxTimedLaunches] = {};
  cudaEvent_t rt_ev[2 * kMaxRounds] = {};
  int rt_n = 0;
  int64_t rt_act[kMaxRounds] = {};
  int kt_n = 0;
  int kt_bpe[kMaxTimedLaunches] = {};
  uint64_t *h_kt = nullptr;
  // The slab workspace and the host arrays strided by its block slots.
  void release_slab() {
    delete ws;
    ws = nullptr;
    for (void *p : {(void *)h_out, (void *)h_sizes, (void *)h_crc, (void *)h_cnt,
                    (void *)h_act, (void *)h_err})
      if (p) cudaFreeHost(p);
    h_out = nullptr;
    h_sizes = nullptr;
    h_crc = nullptr;
    h_cnt = nullptr;
    h_act = nullptr;
    h_err = nullptr;
    h_out_cap = 0;
    slots = 0;
  }
  // (Re)creates them for slabs of up to `blocks` blocks of max_block_bytes.
  void size_slab(int blocks, int64_t max_block_bytes) {
    BZ_CUDA(cudaStreamSynchronize(st));
    release_slab();
    ws = Workspace::create_for(blocks, max_block_bytes, kBatchSlots);
    slots = ws->max_blocks;
    const int S = slots;
    h_out_cap = (size_t)ws->out_words * 4;
    BZ_CUDA(cudaMallocHost((void **)&h_out, h_out_cap));
    BZ_CUDA(cudaMallocHost((void **)&h_sizes, sizeof(int64_t) * 2 * S));
    BZ_CUDA(cudaMallocHost((void **)&h_crc, sizeof(uint32_t) * S));
    BZ_CUDA(cudaMallocHost((void **)&h_cnt, sizeof(int32_t) * 5 * S));
    BZ_CUDA(cudaMallocHost((void **)&h_act, sizeof(int64_t) * S));
    BZ_CUDA(cudaMallocHost((void **)&h_err, sizeof(int32_t)));
    ws->dev.rt_ev = rt_ev;
    ws->dev.rt_n = &rt_n;
    ws->dev.rt_act = rt_act;
    ws->dev.kt_ev = kt_ev;
    ws->dev.kt_n = &kt_n;
    ws->dev.kt_bpe = kt_bpe;
  }
  ~Worker() {
    if (st) cudaStreamSynchronize(st);
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
    for (auto &e : kt_ev)
      if (e) cudaEventDestroy(e);
    for (auto &e : rt_ev)
      if (e) cudaEventDestroy(e);
    if (h_kt) cudaFreeHost(h_kt);
    release_slab();
    if (st) cudaStreamDestroy(st);
  }
};

Compressor::Compressor(const CompressorConfig &cfg) : cfg_(cfg) {
  BZ_CUDA(cudaGetDevice(&device_));
  if (cfg_.slab_blocks < 1) cfg_.slab_blocks = 1;
  if (cfg_.workers < 1) cfg_.workers = 1;
  for (int i = 0; i < cfg_.workers; i++) {
    auto w = std::make_unique<Worker>();
    BZ_CUDA(cudaStreamCreateWithFlags(&w->st, cudaStreamNonBlocking));
    for (auto &e : w->ev) BZ_CUDA(cudaEventCreate(&e));
    for (auto &e : w->kt_ev) BZ_CUDA(cudaEventCreate(&e));
    for (auto &e : w->rt_ev) BZ_CUDA(cudaEventCreate(&e));
    BZ_CUDA(cudaMallocHost((void **)&w->h_kt, 8 * kMaxTimedLaunches));
    workers_.push_back(std::move(w));
  }
}

// Slab workspaces are sized on demand (caller holds the call lock): a call
// of `blocks` blocks needs slabs of at most min(blocks, slab_blocks) blocks,
// so small calls take little device memory.  A call that needs more than
// the workers hold grows every worker's workspace, at least doubling it and
// at most to slab_blocks blocks; the workspaces are then kept for later
// calls.
void Compressor::reserve(int blocks) {
  const int want = std::max(1, std::min(blocks, cfg_.slab_blocks));
  if (slab_capacity_ >= want) return;
  const int nb = std::min(cfg_.slab_blocks, std::max(want, 2 * slab_capacity_));
  slab_capacity_ = 0;  // stays 0 if a (re)allocation fails part way
  for (auto &w : workers_) w->size_slab(nb, cfg_.max_block_bytes);
  slab_capacity_ = nb;
}

Compressor::~Compressor() {
  for (uint32_t *c : arena_chunks_) cudaFree(c);
  if (splice_out_) cudaFree(splice_out_);
  if (splice_meta_) cudaFree(splice_meta_);
}

void Compressor::set_batch_tuning(const std::vector<BatchTune> &table) {
  std::lock_guard<std::mutex> call_lock(call_mu_);
  for (const BatchTune &t : table)
    BZ_REQUIRE(t.max_len > 0 && t.slab_blocks > 0 && t.workers > 0, kErrArg,
               "batch tuning entries must be positive");
  tune_ = table;
  std::sort(tune_.begin(), tune_.end(),
            [](const BatchTune &a, const BatchTune &b) { return a.max_len < b.max_len; });
}

// The tuning entry for blocks of `len` raw bytes: the first whose max_len
// covers it, the last one beyond, the engine's own shape without a table.
Compressor::BatchTune Compressor::tune_for(int len) const {
  if (tune_.empty()) return {len, cfg_.slab_blocks, (int)workers_.size()};
  for (const BatchTune &t : tune_)
    if (len <= t.max_len) return t;
  return tune_.back();
}

// A run of `words` arena words for one slab (caller holds the batch lock):
// the current chunk if it has room, else the next one, allocated once and
// kept for later calls.
uint32_t *Compressor::arena_take(int64_t words, size_t *chunk, int64_t *used, int64_t *base) {
  const int64_t cw = std::max<int64_t>(kArenaChunkWords, words);
  if (*chunk < arena_chunks_.size() && *used + words > arena_chunk_words_[*chunk]) {
    (*chunk)++;
    *used = 0;
  }
  while (*chunk < arena_chunks_.size() && words > arena_chunk_words_[*chunk]) (*chunk)++;
  if (*chunk >= arena_chunks_.size()) {
    uint32_t *p = nullptr;
    BZ_CUDA(cudaMalloc((void **)&p, sizeof(uint32_t) * cw));
    arena_chunks_.push_back(p);
    arena_chunk_words_.push_back(cw);
    *chunk = arena_chunks_.size() - 1;
    *used = 0;
  }
  *base = *used;
  *used += words;
  return arena_chunks_[*chunk];
}

ByteSink::ByteSink(uint8_t *p, size_t c) : data(p), size(0), cap(c), owned(false) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) == cudaSuccess) {
    pinned = a.type == cudaMemoryTypeHost;
    device = a.type == cudaMemoryTypeDevice;
  } else {
    cudaGetLastError();
  }
}

ByteSink::~ByteSink() {
  if (owned) std::free(data);
}

void ByteSink::reserve(size_t c) {
  BZ_REQUIRE(owned || c <= cap, kErrTooLarge, "output buffer too small");
  if (!owned || c <= cap) return;
  // large buffers are mapped lazily: untouched pages cost nothing
  uint8_t *p = (uint8_t *)std::realloc(data, c);
  BZ_REQUIRE(p, kErrAlloc, "host output allocation failed");
  data = p;
  cap = c;
}

uint8_t *ByteSink::release() {
  uint8_t *p = data;
  if (size < cap && size > 0) {
    uint8_t *q = (uint8_t *)std::realloc(p, size);
    if (q) p = q;
  }
  data = nullptr;
  size = cap = 0;
  return p;
}

size_t stream_bound(int64_t n, int64_t nblocks) {
  // header <= 20000 bytes per block (selectors <= 6 bits each, tables);
  // payload <= 17 bits per symbol, symbols <= RLE1 bytes + 1
  return 64 + (size_t)nblocks * 20000 + (size_t)(rle1_bound(n) + nblocks * 16) * kMaxCodeLen / 8;
}

namespace {
// Device sinks: the first bytes of a slab's part share a word with the
// previous slab's last bytes; OR them in (or store them past the end).
__global__ void k_merge_head(uint8_t *dst, uint32_t head, int n, int64_t keep) {
  for (int i = 0; i < n; i++) {
    const uint8_t b = (uint8_t)(head >> (8 * i));
    if (i < keep) dst[i] |= b;
    else dst[i] = b;
  }
}

// The selector's tensor-core kernel bounds every wait; a wait that ran out
// leaves a nonzero error word in the workspace (read back with the sizes).
void check_err_word(const int32_t *h_err) {
  BZ_REQUIRE(*h_err == 0, kErrInternal,
             "learned selector: a tensor-core wait timed out (error word " +
                 std::to_string(*h_err) + ")");
}

}  // namespace

// 48-bit end-of-stream magic then the 32-bit combined CRC, MSB first, then
// padding to a byte (src/compression/compress.cu:366-376).
void put_eos(ByteSink &out, size_t base, int64_t bit, uint32_t crc) {
  const uint64_t magic = 0x177245385090ull;
  auto put = [&](uint64_t v, int nb) {
    for (int k = nb - 1; k >= 0; k--) {
      size_t byte = base + (size_t)(bit >> 3);
      if (byte >= out.size) out.data[out.size++] = 0;
      if ((v >> k) & 1) out.data[byte] |= (uint8_t)(0x80u >> (bit & 7));
      bit++;
    }
  };
  put(magic, 48);
  put(crc, 32);
}

void Compressor::compress(const uint8_t *const *ptrs, const int *lens, int nblocks, int level,
                          ByteSink &out, StageTimes *times) {
  run(ptrs, lens, nblocks, level, false, out, times);
}

void Compressor::compress_device(const uint8_t *const *d_ptrs, const int *lens, int nblocks,
                                 int level, ByteSink &out, StageTimes *times) {
  run(d_ptrs, lens, nblocks, level, true, out, times);
}

void Compressor::compress(const uint8_t *const *ptrs, const int *lens, int nblocks, int level,
                          std::vector<uint8_t> &out, StageTimes *times) {
  ByteSink s;
  compress(ptrs, lens, nblocks, level, s, times);
  out.insert(out.end(), s.data, s.data + s.size);
}

void Compressor::compress_part(const uint8_t *const *ptrs, const int *lens, int nblocks,
                               bool on_device, ByteSink &out, int64_t *bits, uint32_t *crc_fold,
                               StageTimes *times) {
  BZ_REQUIRE(out.device && !out.owned, kErrArg, "a part is written to a device buffer");
  run(ptrs, lens, nblocks, 9, on_device, out, times, true, bits, crc_fold);
}

void Compressor::run(const uint8_t *const *ptrs, const int *lens, int nblocks, int level,
                     bool on_device, ByteSink &out, StageTimes *times, bool part,
                     int64_t *part_bits, uint32_t *part_crc) {
  std::lock_guard<std::mutex> call_lock(call_mu_);
  {
    // room for min(nblocks, slab_blocks) blocks; with an RLE1 cap a block's
    // raw bytes may exceed max_block_bytes and take the raw room of several
    int want = nblocks;
    if (cfg_.m_cap > 0) {
      const int64_t per = align_up(std::max<int64_t>(cfg_.max_block_bytes, 1), 16);
      for (int b = 0; b < nblocks; b++)
        want = (int)std::max<int64_t>(want, (lens[b] + per - 1) / per);
    }
    reserve(want);
  }
  const Workspace &ws0 = *workers_[0]->ws;
  const int64_t raw_max = cfg_.m_cap > 0 ? ws0.max_raw : cfg_.max_block_bytes;
  BZ_REQUIRE(cfg_.m_cap <= rle1_bound(cfg_.max_block_bytes), kErrArg,
             "RLE1 cap above the workspace's block size");
  int64_t ntot = 0;
  for (int b = 0; b < nblocks; b++) {
    BZ_REQUIRE(lens[b] > 0 && lens[b] <= raw_max, kErrArg,
               cfg_.m_cap > 0
                   ? "block of " + std::to_string(lens[b]) +
                         " raw bytes exceeds a slab's raw capacity of " +
                         std::to_string(raw_max) + " bytes (raise slab_blocks)"
                   : std::string("block length outside (0, max_block_bytes]"));
    ntot += lens[b];
  }
  if (level < 1) level = 1;
  if (level > 9) level = 9;
  const size_t base = out.size;
  const size_t bound = stream_bound(ntot, nblocks);
  if (out.owned) out.reserve(base + bound);
  BZ_REQUIRE(base + 14 <= out.cap, kErrTooLarge, "output buffer too small");
  BZ_REQUIRE(!out.device || part, kErrArg, "whole streams are written to host memory");
  if (!part) {
    out.data[base + 0] = 'B';
    out.data[base + 1] = 'Z';
    out.data[base + 2] = 'h';
    out.data[base + 3] = (uint8_t)('0' + level);
    out.size = base + 4;
  }
  const int B = cfg_.slab_blocks;
  // slabs: up to B blocks, fewer where long blocks would overflow a workspace
  std::vector<int> slab_at{0};
  {
    int64_t raw = 0, elems = 0;
    int rt = 0, tiles = 0, gt = 0, cnt = 0;
    for (int b = 0; b < nblocks; b++) {
      const BlockNeeds q = block_needs(lens[b], cfg_.m_cap);
      BZ_REQUIRE(q.raw <= ws0.max_raw && q.raw_tiles <= ws0.max_raw_tiles &&
                     q.elems <= ws0.max_elems && q.tiles <= ws0.max_tiles &&
                     q.group_tiles <= ws0.max_group_tiles,
                 kErrArg, "block larger than a slab");
      if (cnt == B || raw + q.raw > ws0.max_raw || rt + q.raw_tiles > ws0.max_raw_tiles ||
          elems + q.elems > ws0.max_elems || tiles + q.tiles > ws0.max_tiles ||
          gt + q.group_tiles > ws0.max_group_tiles) {
        slab_at.push_back(b);
        raw = elems = 0;
        rt = tiles = gt = cnt = 0;
      }
      raw += q.raw;
      elems += q.elems;
      rt += q.raw_tiles;
      tiles += q.tiles;
      gt += q.group_tiles;
      cnt++;
    }
    if (nblocks > 0) slab_at.push_back(nblocks);
  }
  const int nslabs = (int)slab_at.size() - 1;

  std::mutex mu;
  std::condition_variable cv;
  int next_offset = 0, next_append = 0;
  int64_t bit = part ? 0 : 32;
  uint32_t stream_crc = 0;
  std::exception_ptr err;
  std::atomic<int> next_slab{0};
  StageTimes tsum;

  auto work = [&](Worker &w) {
    BZ_CUDA(cudaSetDevice(device_));
    SlabPlan plan;
    for (;;) {
      {
        std::lock_guard<std::mutex> g(mu);
        if (err) return;
      }
      const int k = next_slab.fetch_add(1);
      if (k >= nslabs) return;
      const int b0 = slab_at[k], nb = slab_at[k + 1] - b0;
      plan.build(lens + b0, nb, cfg_.run_cut, cfg_.m_cap);
      w.ws->upload_plan(plan, w.st);
      const SlabDev &d = w.ws->dev;
      // raw bytes: one copy when the blocks are back to back and 16-aligned
      bool contiguous = true;
      for (int i = 0; i + 1 < nb && contiguous; i++)
        contiguous = ptrs[b0 + i] + lens[b0 + i] == ptrs[b0 + i + 1] && lens[b0 + i] % 16 == 0;
      const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
      if (contiguous) {
        int64_t tot = 0;
        for (int i = 0; i < nb; i++) tot += lens[b0 + i];
        BZ_CUDA(cudaMemcpyAsync(d.raw, ptrs[b0], tot, kind, w.st));
      } else {
        for (int i = 0; i < nb; i++)
          BZ_CUDA(cudaMemcpyAsync(d.raw + plan.raw_off[i], ptrs[b0 + i], lens[b0 + i], kind, w.st));
      }
      const bool tm = times != nullptr && cfg_.time_stages;
      w.ws->dev.kt_on = tm;
      w.kt_n = 0;
      w.rt_n = 0;
      if (tm) BZ_CUDA(cudaMemsetAsync(d.kt_elems, 0, 8 * kMaxTimedLaunches, w.st));
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[0], w.st));
      stage_rle1_crc(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[1], w.st));
      stage_bwt(d, plan.max_m_bound, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[2], w.st));
      stage_mtf(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[3], w.st));
      stage_rle2(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[4], w.st));
      stage_huffman(d, w.st, cfg_.selector, cfg_.plain_passes);
      if (cfg_.tap) mlp::tap_groups(d, *cfg_.tap, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[5], w.st));
      stage_sizes(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[6], w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_sizes, d.hdr_bits, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost,
                              w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_sizes + w.slots, d.pay_bits, sizeof(int64_t) * nb,
                              cudaMemcpyDeviceToHost, w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_crc, d.crc, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost, w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_err, d.err, sizeof(int32_t), cudaMemcpyDeviceToHost, w.st));
      if (times) {
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt, d.m, 4 * nb, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + w.slots, d.s, 4 * nb, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + 2 * w.slots, d.n_sel, 4 * nb, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + 3 * w.slots, d.learned, 4 * nb, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + 4 * w.slots, d.n_groups, 4 * nb, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_act, d.active_sum, 8 * nb, cudaMemcpyDeviceToHost, w.st));
      }
      if (tm && w.kt_n > 0)
        BZ_CUDA(cudaMemcpyAsync(w.h_kt, d.kt_elems, 8 * w.kt_n, cudaMemcpyDeviceToHost, w.st));
      BZ_CUDA(cudaStreamSynchronize(w.st));
      check_err_word(w.h_err);
      int64_t total = 0;
      for (int i = 0; i < nb; i++) total += w.h_sizes[i] + w.h_sizes[w.slots + i];
      if (times) {
        std::lock_guard<std::mutex> g(mu);
        for (int i = 0; i < nb; i++) {
          tsum.blocks++;
          tsum.n += lens[b0 + i];
          tsum.m += w.h_cnt[i];
          tsum.s += w.h_cnt[w.slots + i];
          tsum.g += w.h_cnt[2 * w.slots + i];
          tsum.A += w.h_act[i];
          tsum.bits += w.h_sizes[w.slots + i];
          tsum.learned_blocks += w.h_cnt[3 * w.slots + i];
          tsum.six_table_blocks += w.h_cnt[4 * w.slots + i] == kMaxGroups;
        }
      }
      int64_t start;
      {
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&] { return next_offset == k || err; });
        if (err) return;
        start = bit;
        for (int i = 0; i < nb; i++) stream_crc = ((stream_crc << 1) | (stream_crc >> 31)) ^ w.h_crc[i];
        bit = start + total;
        next_offset++;
        cv.notify_all();
      }
      const int64_t end = start + total;
      const int64_t w0 = start / 32;
      const int64_t nwords = (end + 31) / 32 - w0;
      BZ_REQUIRE(nwords <= w.ws->out_words, kErrInternal, "slab output exceeds buffer");
      const size_t at = base + (size_t)(4 * w0);
      const int64_t nbytes = (end + 7) / 8 - 4 * w0;
      BZ_REQUIRE(at + (size_t)nbytes + 10 <= out.cap, kErrTooLarge, "output buffer too small");
      stage_place(d, start, w0, nwords, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[7], w.st));
      // The slab owns its bytes from 4*w0 + 4 on; its first word is shared
      // with the previous slab's last one and is OR-ed in slab order below.
      const int64_t head = std::min<int64_t>(4, nbytes);
      BZ_CUDA(cudaMemcpyAsync(w.h_out, d.out, head, cudaMemcpyDeviceToHost, w.st));
      if (nbytes > head) {
        if (out.device) {
          BZ_CUDA(cudaMemcpyAsync(out.data + at + head, (const uint8_t *)d.out + head,
                                  nbytes - head, cudaMemcpyDeviceToDevice, w.st));
          BZ_CUDA(cudaStreamSynchronize(w.st));
        } else if (out.pinned) {
          BZ_CUDA(cudaMemcpyAsync(out.data + at + head, (const uint8_t *)d.out + head,
                                  nbytes - head, cudaMemcpyDeviceToHost, w.st));
          BZ_CUDA(cudaStreamSynchronize(w.st));
        } else {
          BZ_CUDA(cudaMemcpyAsync(w.h_out + head, (const uint8_t *)d.out + head, nbytes - head,
                                  cudaMemcpyDeviceToHost, w.st));
          BZ_CUDA(cudaStreamSynchronize(w.st));
          std::memcpy(out.data + at + head, w.h_out + head, nbytes - head);
        }
      } else {
        BZ_CUDA(cudaStreamSynchronize(w.st));
      }
      if (tm) {
        float ms[7];
        for (int q = 0; q < 6; q++) BZ_CUDA(cudaEventElapsedTime(&ms[q], w.ev[q], w.ev[q + 1]));
        BZ_CUDA(cudaEventElapsedTime(&ms[6], w.ev[6], w.ev[7]));
        std::lock_guard<std::mutex> g(mu);
        tsum.rle1 += ms[0];
        tsum.bwt += ms[1];
        tsum.mtf += ms[2];
        tsum.rle2 += ms[3];
        tsum.huffman += ms[4];
        tsum.sizes += ms[5];
        tsum.place += ms[6];
        for (int r = 0; r < w.rt_n; r++) {
          float t = 0;
          BZ_CUDA(cudaEventElapsedTime(&t, w.rt_ev[2 * r], w.rt_ev[2 * r + 1]));
          tsum.round_ms[r] += t;
          tsum.round_active[r] += w.rt_act[r];
        }
        for (int q = 0; q < w.kt_n; q++) {
          if (w.h_kt[q] == 0) continue;  // skipped pass (one digit value only)
          float t = 0;
          BZ_CUDA(cudaEventElapsedTime(&t, w.kt_ev[2 * q], w.kt_ev[2 * q + 1]));
          tsum.scatter_launches++;
          tsum.scatter_ms += t;
          tsum.scatter_bytes += (double)w.h_kt[q] * w.kt_bpe[q];
        }
      }
      {
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&] { return next_append == k || err; });
        if (err) return;
        // bytes [at, out.size) hold the previous slab's tail (<= 4 bytes)
        if (out.device) {
          uint32_t hv = 0;
          for (int64_t i = 0; i < head; i++) hv |= (uint32_t)w.h_out[i] << (8 * i);
          const int64_t keep = (int64_t)out.size > (int64_t)at ? (int64_t)out.size - (int64_t)at : 0;
          k_merge_head<<<1, 1, 0, w.st>>>(out.data + at, hv, (int)head, keep);
          BZ_LAUNCH_CHECK();
          BZ_CUDA(cudaStreamSynchronize(w.st));
        } else {
          for (int64_t i = 0; i < head; i++) {
            if (at + i < out.size) out.data[at + i] |= w.h_out[i];
            else out.data[at + i] = w.h_out[i];
          }
        }
        out.size = at + (size_t)nbytes;
        next_append++;
        cv.notify_all();
      }
    }
  };

  const int nw = std::min<int>((int)workers_.size(), std::max(nslabs, 1));
  std::vector<std::thread> th;
  auto guarded = [&](Worker &w) {
    try {
      work(w);
    } catch (...) {
      std::lock_guard<std::mutex> g(mu);
      if (!err) err = std::current_exception();
      cv.notify_all();
    }
  };
  for (int i = 1; i < nw; i++) th.emplace_back(guarded, std::ref(*workers_[i]));
  if (nw >= 1) guarded(*workers_[0]);
  for (auto &t : th) t.join();
  if (err) {
    out.size = base;
    std::rethrow_exception(err);
  }
  if (part) {
    if (part_bits) *part_bits = bit;
    if (part_crc) *part_crc = stream_crc;
  } else {
    put_eos(out, base, bit, stream_crc);
  }
  if (times) *times = tsum;
}


// ------------------------------------------------------------ batched form
void Compressor::compress_batch(const Item *items, int count, bool on_device, ByteSink &out,
                                std::vector<size_t> &offsets, StageTimes *times) {
  std::lock_guard<std::mutex> call_lock(call_mu_);
  struct Blk {
    int item, k;
    const uint8_t *ptr;
    int len;
    int64_t arena_word = 0, bits = 0;
    const uint32_t *src = nullptr;
    uint32_t crc = 0;
  };
  std::vector<Blk> blks;
  int64_t ntot = 0;
  for (int i = 0; i < count; i++) {
    const Item &it = items[i];
    BZ_REQUIRE(it.n >= 0 && (it.n == 0 || it.ptr), kErrArg, "bad batch item");
    BZ_REQUIRE(it.block_bytes > 0 && it.block_bytes <= cfg_.max_block_bytes, kErrArg,
               "batch item block size outside (0, max_block_bytes]");
    for (int64_t o = 0, k = 0; o < it.n; o += it.block_bytes, k++)
      blks.push_back({i, (int)k, it.ptr + o, (int)std::min<int64_t>(it.block_bytes, it.n - o)});
    ntot += it.n;
  }
  const int nb = (int)blks.size();
  // the work queue: longest blocks first, so slabs hold similar lengths
  std::vector<int> order(nb);
  for (int i = 0; i < nb; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return blks[a].len > blks[b].len; });
  // slabs over the queue: a slab takes up to the tuned block count for its
  // longest (first) block, fewer where the workspace's capacities end
  reserve(nb);
  const Workspace &ws0 = *workers_[0]->ws;
  std::vector<int> slab_at{0};
  {
    int64_t raw = 0, elems = 0;
    int rt = 0, tiles = 0, gt = 0, cnt = 0, cap = 0;
    for (int q = 0; q < nb; q++) {
      const BlockNeeds bn = block_needs(blks[order[q]].len, 0);
      if (cnt > 0 && (cnt == cap || raw + bn.raw > ws0.max_raw || elems + bn.elems > ws0.max_elems ||
                      rt + bn.raw_tiles > ws0.max_raw_tiles || tiles + bn.tiles > ws0.max_tiles ||
                      gt + bn.group_tiles > ws0.max_group_tiles)) {
        slab_at.push_back(q);
        raw = elems = 0;
        rt = tiles = gt = cnt = 0;
      }
      if (cnt == 0) cap = std::min(tune_for(blks[order[q]].len).slab_blocks, ws0.max_blocks);
      raw += bn.raw;
      elems += bn.elems;
      rt += bn.raw_tiles;
      tiles += bn.tiles;
      gt += bn.group_tiles;
      cnt++;
    }
    if (nb > 0) slab_at.push_back(nb);
  }
  const int nslabs = (int)slab_at.size() - 1;
  // worker streams: the tuned count for the byte-weighted median block length
  int tuned_workers = (int)workers_.size();
  if (nb > 0) {
    int64_t half = 0, acc = 0;
    for (const Blk &bk : blks) half += bk.len;
    half /= 2;
    for (int q = nb - 1; q >= 0; q--) {  // shortest first
      acc += blks[order[q]].len;
      if (acc >= half) {
        tuned_workers = tune_for(blks[order[q]].len).workers;
        break;
      }
    }
  }
  // arena: every block's bits, word-aligned, in chunks kept by the engine
  size_t chunk = 0;
  int64_t chunk_used = 0;

  std::mutex mu;
  std::exception_ptr err;
  std::atomic<int> next_slab{0};
  StageTimes tsum;

  auto work = [&](Worker &w) {
    BZ_CUDA(cudaSetDevice(device_));
    SlabPlan plan;
    std::vector<int> lens(w.slots);
    for (;;) {
      {
        std::lock_guard<std::mutex> g(mu);
        if (err) return;
      }
      const int k = next_slab.fetch_add(1);
      if (k >= nslabs) return;
      const int s0 = slab_at[k], ns = slab_at[k + 1] - s0;
      for (int i = 0; i < ns; i++) lens[i] = blks[order[s0 + i]].len;
      plan.build(lens.data(), ns);
      w.ws->upload_plan(plan, w.st);
      const SlabDev &d = w.ws->dev;
      const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
      // one copy per run of blocks that are adjacent both in the source and in
      // the slab (16-byte multiples)
      for (int i = 0; i < ns;) {
        int j = i + 1;
        while (j < ns && blks[order[s0 + j]].ptr == blks[order[s0 + j - 1]].ptr + lens[j - 1] &&
               plan.raw_off[j] == plan.raw_off[j - 1] + lens[j - 1])
          j++;
        const int64_t bytes = plan.raw_off[j - 1] + lens[j - 1] - plan.raw_off[i];
        BZ_CUDA(cudaMemcpyAsync(d.raw + plan.raw_off[i], blks[order[s0 + i]].ptr, bytes, kind,
                                w.st));
        i = j;
      }
      w.ws->dev.kt_on = 0;
      stage_rle1_crc(d, w.st);
      stage_bwt(d, plan.max_m_bound, w.st);
      stage_mtf(d, w.st);
      stage_rle2(d, w.st);
      stage_huffman(d, w.st, cfg_.selector, cfg_.plain_passes);
      if (cfg_.tap) mlp::tap_groups(d, *cfg_.tap, w.st);
      stage_sizes(d, w.st);
      BZ_CUDA(cudaMemcpyAsync(w.h_sizes, d.hdr_bits, sizeof(int64_t) * ns, cudaMemcpyDeviceToHost,
                              w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_sizes + w.slots, d.pay_bits, sizeof(int64_t) * ns,
                              cudaMemcpyDeviceToHost, w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_crc, d.crc, sizeof(uint32_t) * ns, cudaMemcpyDeviceToHost, w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_err, d.err, sizeof(int32_t), cudaMemcpyDeviceToHost, w.st));
      if (times) {
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt, d.m, 4 * ns, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + w.slots, d.s, 4 * ns, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + 2 * w.slots, d.n_sel, 4 * ns, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + 3 * w.slots, d.learned, 4 * ns, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + 4 * w.slots, d.n_groups, 4 * ns, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_act, d.active_sum, 8 * ns, cudaMemcpyDeviceToHost, w.st));
      }
      BZ_CUDA(cudaStreamSynchronize(w.st));
      check_err_word(w.h_err);
      int64_t words = 0;
      int64_t base;
      uint32_t *arena;
      {
        std::lock_guard<std::mutex> g(mu);
        for (int i = 0; i < ns; i++) words += (w.h_sizes[i] + w.h_sizes[w.slots + i] + 31) / 32;
        arena = arena_take(words, &chunk, &chunk_used, &base);
        int64_t at = base;
        for (int i = 0; i < ns; i++) {
          Blk &bk = blks[order[s0 + i]];
          const int64_t bits = w.h_sizes[i] + w.h_sizes[w.slots + i];
          bk.arena_word = at;
          bk.src = arena + at;
          bk.bits = bits;
          bk.crc = w.h_crc[i];
          at += (bits + 31) / 32;
        }
        if (times)
          for (int i = 0; i < ns; i++) {
            tsum.blocks++;
            tsum.n += lens[i];
            tsum.m += w.h_cnt[i];
            tsum.s += w.h_cnt[w.slots + i];
            tsum.g += w.h_cnt[2 * w.slots + i];
            tsum.A += w.h_act[i];
            tsum.bits += w.h_sizes[w.slots + i];
            tsum.learned_blocks += w.h_cnt[3 * w.slots + i];
            tsum.six_table_blocks += w.h_cnt[4 * w.slots + i] == kMaxGroups;
          }
      }
      // block starts (bits) in the arena, staged through the sizes buffer
      for (int i = 0; i < ns; i++) w.h_sizes[i] = blks[order[s0 + i]].arena_word * 32;
      BZ_CUDA(cudaMemcpyAsync(d.blk_start, w.h_sizes, sizeof(int64_t) * ns, cudaMemcpyHostToDevice,
                              w.st));
      stage_place_arena(d, arena, base, words, w.st);
      BZ_CUDA(cudaStreamSynchronize(w.st));
    }
  };

  if (nslabs > 0) {
    const int nw = std::max(1, std::min({(int)workers_.size(), nslabs, tuned_workers}));
    std::vector<std::thread> th;
    auto guarded = [&](Worker &w) {
      try {
        work(w);
      } catch (...) {
        std::lock_guard<std::mutex> g(mu);
        if (!err) err = std::current_exception();
      }
    };
    for (int i = 1; i < nw; i++) th.emplace_back(guarded, std::ref(*workers_[i]));
    guarded(*workers_[0]);
    for (auto &t : th) t.join();
    if (err) std::rethrow_exception(err);
  }

  // stream layout: item i occupies [offsets[i], offsets[i+1]) of the output
  const size_t base = out.size;
  offsets.assign(count + 1, base);
  std::vector<int64_t> first_blk(count + 1, 0);
  for (int i = 0, b = 0; i < count; i++) {
    first_blk[i] = b;
    while (b < nb && blks[b].item == i) b++;
    first_blk[i + 1] = b;
  }
  std::vector<int64_t> h_src(std::max(nb, 1)), h_dst(std::max(nb, 1)), h_bits(std::max(nb, 1));
  std::vector<int64_t> end_bit(count);
  std::vector<uint32_t> scrc(count, 0);
  size_t pos = 0;  // bytes from base
  for (int i = 0; i < count; i++) {
    int64_t bit = 32;
    for (int64_t b = first_blk[i]; b < first_blk[i + 1]; b++) {
      h_src[b] = (int64_t)(uintptr_t)blks[b].src;
      h_dst[b] = (int64_t)pos * 8 + bit;
      h_bits[b] = blks[b].bits;
      bit += blks[b].bits;
      scrc[i] = ((scrc[i] << 1) | (scrc[i] >> 31)) ^ blks[b].crc;
    }
    end_bit[i] = bit;
    offsets[i] = base + pos;
    pos += (size_t)((bit + 80 + 7) / 8);
  }
  offsets[count] = base + pos;
  if (out.owned) out.reserve(base + pos + 8);
  BZ_REQUIRE(base + pos <= out.cap, kErrTooLarge, "output buffer too small");
  const int64_t owords = (int64_t)(pos + 3) / 4 + 1;
  cudaStream_t st = workers_[0]->st;
  // the splice buffers are kept by the engine and grown when a call needs more
  if (owords > splice_out_words_) {
    if (splice_out_) BZ_CUDA(cudaFree(splice_out_));
    splice_out_ = nullptr;
    splice_out_words_ = 0;
    BZ_CUDA(cudaMalloc((void **)&splice_out_, sizeof(uint32_t) * owords));
    splice_out_words_ = owords;
  }
  if (nb > splice_meta_blocks_) {
    if (splice_meta_) BZ_CUDA(cudaFree(splice_meta_));
    splice_meta_ = nullptr;
    splice_meta_blocks_ = 0;
    BZ_CUDA(cudaMalloc((void **)&splice_meta_, sizeof(int64_t) * 3 * std::max(nb, 1)));
    splice_meta_blocks_ = std::max(nb, 1);
  }
  uint32_t *d_out = splice_out_;
  int64_t *d_meta = splice_meta_;
  BZ_CUDA(cudaMemsetAsync(d_out, 0, sizeof(uint32_t) * owords, st));
  BZ_CUDA(cudaMemcpyAsync(d_meta, h_src.data(), 8 * nb, cudaMemcpyHostToDevice, st));
  BZ_CUDA(cudaMemcpyAsync(d_meta + nb, h_dst.data(), 8 * nb, cudaMemcpyHostToDevice, st));
  BZ_CUDA(cudaMemcpyAsync(d_meta + 2 * nb, h_bits.data(), 8 * nb, cudaMemcpyHostToDevice, st));
  launch_splice(d_meta, d_meta + nb, d_meta + 2 * nb, nb, d_out, st);
  BZ_CUDA(cudaMemcpyAsync(out.data + base, d_out, pos, cudaMemcpyDeviceToHost, st));
  BZ_CUDA(cudaStreamSynchronize(st));
  out.size = base + pos;
  // stream headers and end-of-stream markers
  for (int i = 0; i < count; i++) {
    int lvl = items[i].level < 1 ? 1 : (items[i].level > 9 ? 9 : items[i].level);
    uint8_t *p = out.data + offsets[i];
    p[0] = 'B';
    p[1] = 'Z';
    p[2] = 'h';
    p[3] = (uint8_t)('0' + lvl);
    ByteSink view(out.data + offsets[i], offsets[i + 1] - offsets[i]);
    view.size = (size_t)((end_bit[i] + 7) / 8);
    put_eos(view, 0, end_bit[i], scrc[i]);
  }
  if (times) *times = tsum;
}

}  // namespace bz2g
