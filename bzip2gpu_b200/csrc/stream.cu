// Streaming compression (stream.h).
#include "stream.h"

#include <algorithm>
#include <cstring>
#include <vector>

#include "engine.h"

namespace bz2g {

StreamWriter::StreamWriter(Compressor &c, int level, Sink sink)
    : c_(c), level_(std::min(std::max(level, 1), 9)), sink_(std::move(sink)) {}

StreamWriter::~StreamWriter() {
  if (d_part_) cudaFree(d_part_);
  if (d_stage_) cudaFree(d_stage_);
  if (d_meta_) cudaFree(d_meta_);
  if (h_stage_) cudaFreeHost(h_stage_);
}

void StreamWriter::emit(const uint8_t *p, size_t n) {
  if (n == 0) return;
  sink_(p, n);
  bytes_out_ += (int64_t)n;
}

void StreamWriter::add(const uint8_t *const *ptrs, const int *lens, int nblocks, bool on_device) {
  if (!header_done_) {
    const uint8_t hdr[4] = {'B', 'Z', 'h', (uint8_t)('0' + level_)};
    emit(hdr, 4);
    header_done_ = true;
  }
  if (nblocks <= 0) return;
  int64_t n = 0;
  for (int b = 0; b < nblocks; b++) n += lens[b];
  const size_t cap = (stream_bound(n, nblocks) + 16 + 3) / 4 * 4;
  if (cap > part_cap_) {
    if (d_part_) BZ_CUDA(cudaFree(d_part_));
    d_part_ = nullptr;
    part_cap_ = 0;
    BZ_CUDA(cudaMalloc((void **)&d_part_, cap));
    part_cap_ = cap;
  }
  ByteSink part(d_part_, part_cap_);
  int64_t bits = 0;
  uint32_t fold = 0;
  c_.compress_part(ptrs, lens, nblocks, on_device, part, &bits, &fold, nullptr);
  // the splice reads whole words: zero the part's tail up to a word
  const size_t used = (size_t)((bits + 7) / 8);
  const size_t end = (used + 3) / 4 * 4;
  cudaStream_t st = 0;
  if (end > used) BZ_CUDA(cudaMemsetAsync(d_part_ + used, 0, end - used, st));
  // splice at the running phase (pending bits first), in 4 MiB segments
  const int64_t total = pending_bits_ + bits;
  const size_t words = (size_t)((total + 31) / 32 + 1);
  if (words > stage_words_) {
    if (d_stage_) BZ_CUDA(cudaFree(d_stage_));
    d_stage_ = nullptr;
    stage_words_ = 0;
    BZ_CUDA(cudaMalloc((void **)&d_stage_, words * 4));
    stage_words_ = words;
  }
  const int64_t seg = int64_t(1) << 25;
  std::vector<int64_t> src, dst, nb;
  for (int64_t o = 0; o < bits; o += seg) {
    src.push_back((int64_t)(uintptr_t)(d_part_ + o / 8));
    dst.push_back(pending_bits_ + o);
    nb.push_back(std::min<int64_t>(seg, bits - o));
  }
  const size_t ns = src.size();
  if (3 * ns > meta_cap_) {
    if (d_meta_) BZ_CUDA(cudaFree(d_meta_));
    d_meta_ = nullptr;
    meta_cap_ = 0;
    BZ_CUDA(cudaMalloc((void **)&d_meta_, 3 * std::max<size_t>(ns, 1) * 8));
    meta_cap_ = 3 * std::max<size_t>(ns, 1);
  }
  BZ_CUDA(cudaMemsetAsync(d_stage_, 0, words * 4, st));
  if (ns > 0) {
    BZ_CUDA(cudaMemcpyAsync(d_meta_, src.data(), 8 * ns, cudaMemcpyHostToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d_meta_ + ns, dst.data(), 8 * ns, cudaMemcpyHostToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d_meta_ + 2 * ns, nb.data(), 8 * ns, cudaMemcpyHostToDevice, st));
    launch_splice(d_meta_, d_meta_ + ns, d_meta_ + 2 * ns, (int)ns, d_stage_, st);
  }
  const size_t out_bytes = (size_t)((total + 7) / 8);
  if (out_bytes + 8 > h_stage_cap_) {
    if (h_stage_) BZ_CUDA(cudaFreeHost(h_stage_));
    h_stage_ = nullptr;
    h_stage_cap_ = 0;
    BZ_CUDA(cudaMallocHost((void **)&h_stage_, out_bytes + 8));
    h_stage_cap_ = out_bytes + 8;
  }
  BZ_CUDA(cudaMemcpyAsync(h_stage_, d_stage_, out_bytes, cudaMemcpyDeviceToHost, st));
  BZ_CUDA(cudaStreamSynchronize(st));
  if (out_bytes > 0) h_stage_[0] |= pending_;
  const size_t full = (size_t)(total / 8);
  emit(h_stage_, full);
  pending_bits_ = (int)(total % 8);
  pending_ = pending_bits_ ? h_stage_[full] : 0;
  const int k = nblocks % 32;
  crc_ = (k ? ((crc_ << k) | (crc_ >> (32 - k))) : crc_) ^ fold;
}

void StreamWriter::finish() {
  if (!header_done_) {
    const uint8_t hdr[4] = {'B', 'Z', 'h', (uint8_t)('0' + level_)};
    emit(hdr, 4);
    header_done_ = true;
  }
  uint8_t buf[16] = {0};
  ByteSink tail(buf, sizeof buf);
  buf[0] = pending_;
  tail.size = pending_bits_ ? 1 : 0;
  put_eos(tail, 0, pending_bits_, crc_);
  emit(buf, tail.size);
  pending_ = 0;
  pending_bits_ = 0;
}

}  // namespace bz2g
