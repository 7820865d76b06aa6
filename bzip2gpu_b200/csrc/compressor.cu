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

namespace bz2g {

struct Compressor::Worker {
  Workspace *ws = nullptr;
  cudaStream_t st = nullptr;
  uint8_t *h_out = nullptr;
  size_t h_out_cap = 0;
  int64_t *h_sizes = nullptr;  // [2 * max_blocks] hdr, pay
  int32_t *h_cnt = nullptr;    // [3 * max_blocks] m, s, n_sel
  int64_t *h_act = nullptr;    // [max_blocks] A
  uint32_t *h_crc = nullptr;
  cudaEvent_t ev[8] = {};
  ~Worker() {
    if (st) cudaStreamSynchronize(st);
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
    delete ws;
    if (h_out) cudaFreeHost(h_out);
    if (h_sizes) cudaFreeHost(h_sizes);
    if (h_crc) cudaFreeHost(h_crc);
    if (h_cnt) cudaFreeHost(h_cnt);
    if (h_act) cudaFreeHost(h_act);
    if (st) cudaStreamDestroy(st);
  }
};

Compressor::Compressor(const CompressorConfig &cfg) : cfg_(cfg) {
  BZ_CUDA(cudaGetDevice(&device_));
  if (cfg_.slab_blocks < 1) cfg_.slab_blocks = 1;
  if (cfg_.workers < 1) cfg_.workers = 1;
  for (int i = 0; i < cfg_.workers; i++) {
    auto w = std::make_unique<Worker>();
    w->ws = Workspace::create_for(cfg_.slab_blocks, cfg_.max_block_bytes);
    BZ_CUDA(cudaStreamCreateWithFlags(&w->st, cudaStreamNonBlocking));
    w->h_out_cap = (size_t)w->ws->out_words * 4;
    BZ_CUDA(cudaMallocHost((void **)&w->h_out, w->h_out_cap));
    BZ_CUDA(cudaMallocHost((void **)&w->h_sizes, sizeof(int64_t) * 2 * cfg_.slab_blocks));
    BZ_CUDA(cudaMallocHost((void **)&w->h_crc, sizeof(uint32_t) * cfg_.slab_blocks));
    BZ_CUDA(cudaMallocHost((void **)&w->h_cnt, sizeof(int32_t) * 3 * cfg_.slab_blocks));
    BZ_CUDA(cudaMallocHost((void **)&w->h_act, sizeof(int64_t) * cfg_.slab_blocks));
    for (auto &e : w->ev) BZ_CUDA(cudaEventCreate(&e));
    workers_.push_back(std::move(w));
  }
}

Compressor::~Compressor() = default;

void append_eos(std::vector<uint8_t> &out, int64_t bit, uint32_t crc) {
  // 48-bit end-of-stream magic then the 32-bit combined CRC, MSB first
  // (src/compression/compress.cu:366-375).
  const uint64_t magic = 0x177245385090ull;
  auto put = [&](uint64_t v, int nb) {
    for (int k = nb - 1; k >= 0; k--) {
      size_t byte = (size_t)(bit >> 3);
      if (byte >= out.size()) out.push_back(0);
      if ((v >> k) & 1) out[byte] |= (uint8_t)(0x80u >> (bit & 7));
      bit++;
    }
  };
  put(magic, 48);
  put(crc, 32);
}

void Compressor::compress(const uint8_t *const *ptrs, const int *lens, int nblocks, int level,
                          std::vector<uint8_t> &out, StageTimes *times) {
  run(ptrs, lens, nblocks, level, false, out, times);
}

void Compressor::compress_device(const uint8_t *const *d_ptrs, const int *lens, int nblocks,
                                 int level, std::vector<uint8_t> &out, StageTimes *times) {
  run(d_ptrs, lens, nblocks, level, true, out, times);
}

void Compressor::run(const uint8_t *const *ptrs, const int *lens, int nblocks, int level,
                     bool on_device, std::vector<uint8_t> &out, StageTimes *times) {
  for (int b = 0; b < nblocks; b++)
    BZ_REQUIRE(lens[b] > 0 && lens[b] <= cfg_.max_block_bytes, kErrArg,
               "block length outside (0, max_block_bytes]");
  if (level < 1) level = 1;
  if (level > 9) level = 9;
  const size_t base = out.size();
  out.push_back('B');
  out.push_back('Z');
  out.push_back('h');
  out.push_back((uint8_t)('0' + level));
  const int B = cfg_.slab_blocks;
  const int nslabs = (nblocks + B - 1) / B;

  std::mutex mu;
  std::condition_variable cv;
  int next_offset = 0, next_append = 0;
  int64_t bit = 32;
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
      const int b0 = k * B, nb = std::min(B, nblocks - b0);
      plan.build(lens + b0, nb);
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
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[0], w.st));
      stage_rle1_crc(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[1], w.st));
      stage_bwt(d, plan.max_m_bound, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[2], w.st));
      stage_mtf(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[3], w.st));
      stage_rle2(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[4], w.st));
      stage_huffman(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[5], w.st));
      stage_sizes(d, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[6], w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_sizes, d.hdr_bits, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost,
                              w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_sizes + B, d.pay_bits, sizeof(int64_t) * nb,
                              cudaMemcpyDeviceToHost, w.st));
      BZ_CUDA(cudaMemcpyAsync(w.h_crc, d.crc, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost, w.st));
      if (times) {
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt, d.m, 4 * nb, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + B, d.s, 4 * nb, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_cnt + 2 * B, d.n_sel, 4 * nb, cudaMemcpyDeviceToHost, w.st));
        BZ_CUDA(cudaMemcpyAsync(w.h_act, d.active_sum, 8 * nb, cudaMemcpyDeviceToHost, w.st));
      }
      BZ_CUDA(cudaStreamSynchronize(w.st));
      int64_t total = 0;
      for (int i = 0; i < nb; i++) total += w.h_sizes[i] + w.h_sizes[B + i];
      if (times) {
        std::lock_guard<std::mutex> g(mu);
        for (int i = 0; i < nb; i++) {
          tsum.blocks++;
          tsum.n += lens[b0 + i];
          tsum.m += w.h_cnt[i];
          tsum.s += w.h_cnt[B + i];
          tsum.g += w.h_cnt[2 * B + i];
          tsum.A += w.h_act[i];
          tsum.bits += w.h_sizes[B + i];
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
      stage_place(d, start, w0, nwords, w.st);
      if (tm) BZ_CUDA(cudaEventRecord(w.ev[7], w.st));
      const int64_t nbytes = (end + 7) / 8 - 4 * w0;
      BZ_CUDA(cudaMemcpyAsync(w.h_out, d.out, nbytes, cudaMemcpyDeviceToHost, w.st));
      BZ_CUDA(cudaStreamSynchronize(w.st));
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
      }
      {
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&] { return next_append == k || err; });
        if (err) return;
        const size_t at = base + (size_t)(4 * w0);
        size_t ov = out.size() > at ? out.size() - at : 0;
        ov = std::min<size_t>(ov, (size_t)nbytes);
        for (size_t i = 0; i < ov; i++) out[at + i] |= w.h_out[i];
        out.insert(out.end(), w.h_out + ov, w.h_out + nbytes);
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
    out.resize(base);
    std::rethrow_exception(err);
  }
  // the stream's byte vector relative to `base`
  std::vector<uint8_t> tail;
  if (base == 0) {
    append_eos(out, bit, stream_crc);
  } else {
    tail.assign(out.begin() + base, out.end());
    append_eos(tail, bit, stream_crc);
    out.resize(base);
    out.insert(out.end(), tail.begin(), tail.end());
  }
  if (times) *times = tsum;
}

}  // namespace bz2g
