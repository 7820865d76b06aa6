// C-ABI entry points (include/bz2g.h).  Per-stage calls run the slab kernels
// on a one-block slab whose workspace is sized for the call.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/bz2g.h"
#include "compressor.h"
#include "engine.h"
#include "selector.h"
#include "split.h"
#include "stream.h"
#include "../../include/io.h"

namespace bz2g {
namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

template <typename F>
int guard(F &&f) {
  try {
    f();
    g_last_error.clear();
    return BZ2G_OK;
  } catch (const Error &e) {
    return fail(e.code, e.what());
  } catch (const std::bad_alloc &) {
    return fail(BZ2G_ERR_ALLOC, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(BZ2G_ERR_INTERNAL, e.what());
  }
}

__global__ void k_present(const uint8_t *in, int n, uint32_t *present) {
  __shared__ uint32_t p[8];
  if (threadIdx.x < 8) p[threadIdx.x] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicOr(&p[in[i] >> 5], 1u << (in[i] & 31));
  __syncthreads();
  if (threadIdx.x < 8 && p[threadIdx.x]) atomicOr(&present[threadIdx.x], p[threadIdx.x]);
}

__global__ void k_histogram(const uint16_t *syms, int s, int32_t *freq) {
  __shared__ int h[kMaxAlpha];
  for (int i = threadIdx.x; i < kMaxAlpha; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s; i += gridDim.x * blockDim.x) {
    int v = syms[i];
    if (v < kMaxAlpha) atomicAdd(&h[v], 1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kMaxAlpha; i += blockDim.x)
    if (h[i]) atomicAdd(&freq[i], h[i]);
}

__global__ void k_set_block(int32_t *arr, int v) { arr[0] = v; }

cudaStream_t S(void *p) { return reinterpret_cast<cudaStream_t>(p); }

// One-block slab sized for `n` raw bytes.
struct OneBlock {
  std::unique_ptr<Workspace> ws;
  SlabPlan plan;
  OneBlock(int n, cudaStream_t st) {
    ws.reset(Workspace::create_for(1, std::max(n, 1)));
    int len = std::max(n, 1);
    plan.build(&len, 1);
    ws->upload_plan(plan, st);
  }
  const SlabDev &d() const { return ws->dev; }
};

void set_int(int32_t *dst, int v, cudaStream_t st) {
  k_set_block<<<1, 1, 0, st>>>(dst, v);
  BZ_LAUNCH_CHECK();
}

// Engines for the whole-stream calls, per device and configuration.
struct EngineKey {
  int dev, slab, workers;
  int64_t maxb;
  bool operator<(const EngineKey &o) const {
    return std::tie(dev, slab, workers, maxb) < std::tie(o.dev, o.slab, o.workers, o.maxb);
  }
};
std::mutex g_eng_mu;
std::map<EngineKey, std::unique_ptr<Compressor>> g_engines;
int g_slab = 384, g_workers = 4;
std::vector<Compressor::BatchTune> g_batch_tune;  // batched form, by block length
bool g_timing = false;
thread_local StageTimes g_last_stats;

// Learned table selector: packed weights per device and the selector mode of
// the whole-stream calls (0 = the reference's plain selector, 1 = learned,
// 2 = the plain selector with one selection pass, a measurement baseline).
std::mutex g_sel_mu;
std::map<int, uint8_t *> g_sel_packed;
int g_sel_mode = 0;

int current_passes() {
  std::lock_guard<std::mutex> g(g_sel_mu);
  return g_sel_mode == 2 ? 1 : kIters;
}

const uint8_t *current_selector() {
  std::lock_guard<std::mutex> g(g_sel_mu);
  if (g_sel_mode != 1) return nullptr;
  int dev = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  auto it = g_sel_packed.find(dev);
  BZ_REQUIRE(it != g_sel_packed.end(), kErrArg,
             "learned selector enabled but no weights loaded on this device");
  return it->second;
}

// Packed weights from fp32 parameters in device memory (temporary buffer).
uint8_t *pack_params(const float *d_params, cudaStream_t st) {
  uint8_t *packed = nullptr;
  BZ_CUDA(cudaMallocAsync((void **)&packed, mlp::kPackedBytes, st));
  mlp::pack(d_params, packed, st);
  return packed;
}

// The device's engine if its shape matches and its blocks are large enough;
// otherwise a new one (at least 900,000-byte blocks) replaces it.
Compressor &engine_for(int64_t block_bytes) {
  int dev = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_eng_mu);
  for (auto &e : g_engines)
    if (e.first.dev == dev && e.first.slab == g_slab && e.first.workers == g_workers &&
        e.first.maxb >= block_bytes)
      return *e.second;
  int64_t maxb = std::max<int64_t>(block_bytes, 900000);
  for (auto i = g_engines.begin(); i != g_engines.end();) {
    if (i->first.dev == dev) {
      maxb = std::max<int64_t>(maxb, i->first.maxb);
      i = g_engines.erase(i);
    } else {
      ++i;
    }
  }
  CompressorConfig cfg;
  cfg.slab_blocks = g_slab;
  cfg.workers = g_workers;
  cfg.max_block_bytes = maxb;
  auto c = std::make_unique<Compressor>(cfg);
  Compressor &ref = *c;
  g_engines[EngineKey{dev, g_slab, g_workers, maxb}] = std::move(c);
  return ref;
}

// Per-call settings of an engine: timing, selector, and the block format
// (run cut 259 and raw-size blocks, or 255 and RLE1 bytes capped at m_cap).
void set_format(Compressor &c, int run_cut = 259, int64_t m_cap = 0) {
  auto &cfg = const_cast<CompressorConfig &>(c.config());
  cfg.time_stages = g_timing;
  cfg.selector = current_selector();
  cfg.plain_passes = current_passes();
  cfg.run_cut = run_cut;
  cfg.m_cap = m_cap;
}

}  // namespace

Compressor &default_engine(int64_t max_block_bytes) {
  Compressor &c = engine_for(std::max<int64_t>(max_block_bytes, 1));
  set_format(c);
  return c;
}

namespace {

// bzip2 1.0.8's blocks: the split runs on the device copy of the input.
void compress_bzip2(const uint8_t *in, size_t n, int level, bool on_device, ByteSink &out) {
  level = std::min(std::max(level, 1), 9);
  cudaStream_t st = nullptr;
  BZ_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  uint8_t *staged = nullptr;
  struct Cleanup {
    cudaStream_t st;
    uint8_t **staged;
    ~Cleanup() {
      if (*staged) cudaFree(*staged);
      cudaStreamDestroy(st);
    }
  } cleanup{st, &staged};
  const uint8_t *d = in;
  if (!on_device && n > 0) {
    BZ_CUDA(cudaMalloc((void **)&staged, n));
    BZ_CUDA(cudaMemcpyAsync(staged, in, n, cudaMemcpyHostToDevice, st));
    d = staged;
  }
  const std::vector<int64_t> ends = bzip2_split(d, (int64_t)n, level, st);
  std::vector<const uint8_t *> ptrs(ends.size());
  std::vector<int> lens(ends.size());
  int64_t at = 0;
  for (size_t b = 0; b < ends.size(); b++) {
    ptrs[b] = d + at;
    lens[b] = (int)(ends[b] - at);
    at = ends[b];
  }
  Compressor &c = engine_for(900000);
  set_format(c, 255, 100000LL * level);
  g_last_stats = StageTimes();
  c.compress_device(ptrs.data(), lens.data(), (int)ptrs.size(), level, out, &g_last_stats);
}

void compress_any(const uint8_t *in, size_t n, int level, int block_bytes, bool on_device,
                  ByteSink &out) {
  BZ_REQUIRE(n == 0 || in != nullptr, kErrArg, "null input");
  if (block_bytes == BZ2G_BZIP2_BLOCKS) return compress_bzip2(in, n, level, on_device, out);
  BZ_REQUIRE(block_bytes > 0 && block_bytes <= (1 << 24), kErrArg,
             "block_bytes must be in (0, 16 MiB], or BZ2G_BZIP2_BLOCKS");
  const int64_t nb = ((int64_t)n + block_bytes - 1) / block_bytes;
  std::vector<const uint8_t *> ptrs(nb);
  std::vector<int> lens(nb);
  for (int64_t b = 0; b < nb; b++) {
    ptrs[b] = in + b * (int64_t)block_bytes;
    lens[b] = (int)std::min<int64_t>(block_bytes, (int64_t)n - b * (int64_t)block_bytes);
  }
  Compressor &c = engine_for(std::max<int64_t>(block_bytes, 1));
  set_format(c, 259, 0);
  g_last_stats = StageTimes();
  if (on_device)
    c.compress_device(ptrs.data(), lens.data(), (int)nb, level, out, &g_last_stats);
  else
    c.compress(ptrs.data(), lens.data(), (int)nb, level, out, &g_last_stats);
}

}  // namespace

// Lets other translation units report through bz2g_last_error().
void set_last_error(const std::string &msg) { g_last_error = msg; }

}  // namespace bz2g

using namespace bz2g;

extern "C" {

const char *bz2g_last_error(void) { return g_last_error.c_str(); }
int bz2g_version(void) { return 1; }

size_t bz2g_rle1_bound(size_t n) { return (size_t)rle1_bound((int64_t)n); }

size_t bz2g_compress_bound(size_t n, int block_bytes) {
  if (block_bytes == BZ2G_BZIP2_BLOCKS)
    return stream_bound((int64_t)n, bzip2_split_max_blocks((int64_t)n, 1));
  if (block_bytes <= 0) block_bytes = 900000;
  size_t nb = (n + block_bytes - 1) / block_bytes;
  return stream_bound((int64_t)n, (int64_t)nb);
}

int bz2g_set_engine(int slab_blocks, int workers) {
  return guard([&] {
    BZ_REQUIRE(slab_blocks >= 0 && workers >= 0, kErrArg, "negative engine shape");
    std::lock_guard<std::mutex> g(g_eng_mu);
    if (slab_blocks > 0) g_slab = slab_blocks;
    if (workers > 0) g_workers = workers;
  });
}

int bz2g_get_engine(int *slab_blocks, int *workers) {
  return guard([&] {
    BZ_REQUIRE(slab_blocks && workers, kErrArg, "null output pointer");
    std::lock_guard<std::mutex> g(g_eng_mu);
    *slab_blocks = g_slab;
    *workers = g_workers;
  });
}

int bz2g_compress(const uint8_t *in, size_t n, int level, int block_bytes, uint8_t **out,
                  size_t *out_len) {
  return guard([&] {
    BZ_REQUIRE(out && out_len, kErrArg, "null output pointer");
    ByteSink s;
    compress_any(in, n, level, block_bytes, false, s);
    *out_len = s.size;
    *out = s.release();
  });
}

int bz2g_compress_device(const uint8_t *d_in, size_t n, int level, int block_bytes,
                         uint8_t **out, size_t *out_len) {
  return guard([&] {
    BZ_REQUIRE(out && out_len, kErrArg, "null output pointer");
    ByteSink s;
    compress_any(d_in, n, level, block_bytes, true, s);
    *out_len = s.size;
    *out = s.release();
  });
}

int bz2g_compress_into(const uint8_t *in, size_t n, int level, int block_bytes, uint8_t *out,
                       size_t cap, size_t *out_len) {
  return guard([&] {
    BZ_REQUIRE(out && out_len, kErrArg, "null output pointer");
    ByteSink s(out, cap);
    compress_any(in, n, level, block_bytes, false, s);
    *out_len = s.size;
  });
}

int bz2g_compress_device_into(const uint8_t *d_in, size_t n, int level, int block_bytes,
                              uint8_t *out, size_t cap, size_t *out_len) {
  return guard([&] {
    BZ_REQUIRE(out && out_len, kErrArg, "null output pointer");
    ByteSink s(out, cap);
    compress_any(d_in, n, level, block_bytes, true, s);
    *out_len = s.size;
  });
}

void bz2g_free(void *p) { std::free(p); }

int bz2g_bzip2_split(const uint8_t *d_in, size_t n, int level, int64_t *ends, size_t cap,
                     size_t *count, void *stream) {
  return guard([&] {
    BZ_REQUIRE(count && (n == 0 || d_in) && (cap == 0 || ends), kErrArg, "bad arguments");
    const std::vector<int64_t> e = bzip2_split(d_in, (int64_t)n, level, S(stream));
    *count = e.size();
    std::memcpy(ends, e.data(), sizeof(int64_t) * std::min(cap, e.size()));
  });
}

size_t bz2g_bzip2_split_bound(size_t n, int level) {
  return (size_t)bzip2_split_max_blocks((int64_t)n, std::min(std::max(level, 1), 9));
}

size_t bz2g_compress_batch_bound(int count, const size_t *sizes, const int *levels,
                                 const int *block_bytes) {
  size_t tot = 0;
  for (int i = 0; i < count; i++) {
    int bb = block_bytes && block_bytes[i] > 0 ? block_bytes[i]
                                               : 100000 * std::min(std::max(levels[i], 1), 9);
    size_t nb = (sizes[i] + bb - 1) / bb;
    tot += stream_bound((int64_t)sizes[i], (int64_t)nb);
  }
  return tot + 64;
}

int bz2g_compress_batch(int count, const uint8_t *const *inputs, const size_t *sizes,
                        const int *levels, const int *block_bytes, int on_device, uint8_t *out,
                        size_t cap, size_t *offsets) {
  return guard([&] {
    BZ_REQUIRE(count >= 0 && (count == 0 || (inputs && sizes && levels)) && out && offsets,
               kErrArg, "bad arguments");
    std::vector<Compressor::Item> items(count);
    int64_t maxb = 1;
    for (int i = 0; i < count; i++) {
      const int lvl = std::min(std::max(levels[i], 1), 9);
      const int bb = block_bytes && block_bytes[i] > 0 ? block_bytes[i] : 100000 * lvl;
      BZ_REQUIRE(bb <= (1 << 24), kErrArg, "block_bytes above 16 MiB");
      items[i] = {inputs[i], (int64_t)sizes[i], lvl, bb};
      maxb = std::max<int64_t>(maxb, bb);
    }
    Compressor &c = engine_for(maxb);
    ByteSink sink(out, cap);
    std::vector<size_t> offs;
    g_last_stats = StageTimes();
    set_format(c);
    {
      std::vector<Compressor::BatchTune> tune;
      {
        std::lock_guard<std::mutex> g(g_eng_mu);
        tune = g_batch_tune;
      }
      c.set_batch_tuning(tune);
    }
    c.compress_batch(items.data(), count, on_device != 0, sink, offs, &g_last_stats);
    for (int i = 0; i <= count; i++) offsets[i] = offs[i];
  });
}

int bz2g_set_batch_tuning(int n, const int *max_block_len, const int *slab_blocks,
                          const int *workers) {
  return guard([&] {
    BZ_REQUIRE(n >= 0 && (n == 0 || (max_block_len && slab_blocks && workers)), kErrArg,
               "bad arguments");
    std::vector<Compressor::BatchTune> t(n);
    for (int i = 0; i < n; i++) {
      BZ_REQUIRE(max_block_len[i] > 0 && slab_blocks[i] > 0 && workers[i] > 0, kErrArg,
                 "batch tuning entries must be positive");
      t[i] = {max_block_len[i], slab_blocks[i], workers[i]};
    }
    std::lock_guard<std::mutex> g(g_eng_mu);
    g_batch_tune = t;
  });
}

int bz2g_set_timing(int on) {
  std::lock_guard<std::mutex> g(g_eng_mu);
  g_timing = on != 0;
  return BZ2G_OK;
}

int bz2g_last_stats(double *out, int n) {
  const StageTimes &t = g_last_stats;
  const double v[] = {(double)t.blocks, (double)t.n,   (double)t.m,  (double)t.A,
                      (double)t.s,      (double)t.g,   (double)t.bits, t.rle1,
                      t.bwt,            t.mtf,         t.rle2,       t.huffman,
                      t.sizes,          t.place,       (double)t.scatter_launches,
                      t.scatter_ms,     t.scatter_bytes, (double)t.learned_blocks,
                      (double)t.six_table_blocks};
  const int k = (int)(sizeof(v) / sizeof(v[0]));
  for (int i = 0; i < n && i < k; i++) out[i] = v[i];
  return k;
}

int bz2g_last_round_stats(double *out, int n) {
  const StageTimes &t = g_last_stats;
  int rounds = 0;
  for (int r = 0; r < kMaxRounds; r++)
    if (t.round_ms[r] > 0 || t.round_active[r] > 0) rounds = r + 1;
  for (int r = 0; r < rounds && 3 * r + 2 < n; r++) {
    out[3 * r] = r;
    out[3 * r + 1] = (double)t.round_active[r];
    out[3 * r + 2] = t.round_ms[r];
  }
  return rounds;
}

int64_t bz2g_launch_count(void) { return launch_count(); }

int bz2g_rle1(const uint8_t *d_in, int n, uint8_t *d_out, int *m, void *stream) {
  return guard([&] {
    BZ_REQUIRE(n >= 0 && m, kErrArg, "bad arguments");
    if (n == 0) {
      *m = 0;
      return;
    }
    BZ_REQUIRE(d_in && d_out, kErrArg, "null device pointer");
    cudaStream_t st = S(stream);
    OneBlock ob(n, st);
    const SlabDev &d = ob.d();
    BZ_CUDA(cudaMemcpyAsync(d.raw, d_in, n, cudaMemcpyDeviceToDevice, st));
    stage_rle1_crc(d, st);
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.m, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    const int mm = d.h_flags[0];
    BZ_CUDA(cudaMemcpyAsync(d_out, d.rle1, mm, cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    *m = mm;
  });
}

int bz2g_crc32(const uint8_t *d_in, size_t n, uint32_t *crc, void *stream) {
  return guard([&] {
    BZ_REQUIRE(crc, kErrArg, "null crc pointer");
    BZ_REQUIRE(n < (size_t)1 << 30, kErrTooLarge, "crc input above 1 GiB");
    if (n == 0) {
      *crc = 0;
      return;
    }
    cudaStream_t st = S(stream);
    OneBlock ob((int)n, st);
    const SlabDev &d = ob.d();
    BZ_CUDA(cudaMemcpyAsync(d.raw, d_in, n, cudaMemcpyDeviceToDevice, st));
    launch_crc_only(d, st);
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.crc, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    *crc = (uint32_t)d.h_flags[0];
  });
}

int bz2g_bwt(const uint8_t *d_in, int m, int32_t *d_sa, void *stream) {
  return guard([&] {
    BZ_REQUIRE(m >= 0, kErrArg, "negative length");
    if (m == 0) return;
    BZ_REQUIRE(d_in && d_sa, kErrArg, "null device pointer");
    cudaStream_t st = S(stream);
    OneBlock ob(m, st);
    const SlabDev &d = ob.d();
    BZ_CUDA(cudaMemcpyAsync(d.rle1, d_in, m, cudaMemcpyDeviceToDevice, st));
    set_int(d.m, m, st);
    stage_bwt(d, (int)rle1_bound(m), st);
    BZ_CUDA(cudaMemcpyAsync(d_sa, d.sa, sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaStreamSynchronize(st));
  });
}

int bz2g_mtf(const uint8_t *d_orig, const int32_t *d_sa, int m, uint8_t *d_out, int *orig_ptr,
             uint8_t *present, int *n_in_use, void *stream) {
  return guard([&] {
    BZ_REQUIRE(m >= 0, kErrArg, "negative length");
    if (m == 0) {
      if (n_in_use) *n_in_use = 0;
      return;
    }
    BZ_REQUIRE(d_orig && d_sa && d_out, kErrArg, "null device pointer");
    cudaStream_t st = S(stream);
    OneBlock ob(m, st);
    const SlabDev &d = ob.d();
    BZ_CUDA(cudaMemcpyAsync(d.rle1, d_orig, m, cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d.sa, d_sa, sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, st));
    set_int(d.m, m, st);
    set_int(d.orig_ptr, m, st);
    stage_mtf(d, st);
    BZ_CUDA(cudaMemcpyAsync(d_out, d.mtf, m, cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.orig_ptr, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(d.h_flags + 1, d.n_in_use, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(d.h_flags + 2, d.present, 32, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    if (orig_ptr) *orig_ptr = d.h_flags[0];
    if (n_in_use) *n_in_use = d.h_flags[1];
    if (present) {
      const uint32_t *pw = reinterpret_cast<const uint32_t *>(d.h_flags + 2);
      for (int c = 0; c < 256; c++) present[c] = (pw[c >> 5] >> (c & 31)) & 1u;
    }
  });
}

int bz2g_symbols_table(const uint8_t *d_in, int n, uint8_t *table, int *count, void *stream) {
  return guard([&] {
    BZ_REQUIRE(n >= 0 && table && count, kErrArg, "bad arguments");
    cudaStream_t st = S(stream);
    uint32_t *pres = nullptr;
    BZ_CUDA(cudaMallocAsync((void **)&pres, 32, st));
    BZ_CUDA(cudaMemsetAsync(pres, 0, 32, st));
    if (n > 0) {
      int grid = std::min((n + 255) / 256, 1184);
      k_present<<<grid, 256, 0, st>>>(d_in, n, pres);
      BZ_LAUNCH_CHECK();
    }
    uint32_t h[8];
    BZ_CUDA(cudaMemcpyAsync(h, pres, 32, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaFreeAsync(pres, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    int c = 0;
    for (int v = 0; v < 256; v++)
      if ((h[v >> 5] >> (v & 31)) & 1u) table[c++] = (uint8_t)v;
    *count = c;
  });
}

int bz2g_rle2(const uint8_t *d_in, int m, int table_size, uint16_t *d_out, uint32_t *d_out_len,
              void *stream) {
  return guard([&] {
    BZ_REQUIRE(m >= 0 && d_out_len, kErrArg, "bad arguments");
    cudaStream_t st = S(stream);
    if (m == 0) {
      BZ_CUDA(cudaMemsetAsync(d_out_len, 0, sizeof(uint32_t), st));
      return;
    }
    BZ_REQUIRE(d_in && d_out, kErrArg, "null device pointer");
    BZ_REQUIRE(table_size >= 0 && table_size <= 256, kErrArg, "table_size outside [0, 256]");
    OneBlock ob(m, st);
    const SlabDev &d = ob.d();
    BZ_CUDA(cudaMemcpyAsync(d.mtf, d_in, m, cudaMemcpyDeviceToDevice, st));
    set_int(d.m, m, st);
    set_int(d.n_in_use, table_size, st);
    stage_rle2(d, st);
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.s, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    const int s = d.h_flags[0];
    BZ_CUDA(cudaMemcpyAsync(d_out, d.rle2, sizeof(uint16_t) * s, cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d_out_len, d.s, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaStreamSynchronize(st));
  });
}

int bz2g_huffman_build(const uint16_t *d_syms, int s, int n_in_use, uint8_t *len, int32_t *code,
                       uint8_t *selectors, int *n_selectors, int *n_groups, void *stream) {
  return guard([&] {
    BZ_REQUIRE(s > 0 && d_syms && len && code && selectors && n_groups, kErrArg,
               "bad arguments");
    BZ_REQUIRE(n_in_use >= 0 && n_in_use <= 256, kErrArg, "n_in_use outside [0, 256]");
    cudaStream_t st = S(stream);
    // capacity: s symbols need an element layout of at least s entries
    OneBlock ob(s, st);
    const SlabDev &d = ob.d();
    BZ_CUDA(cudaMemcpyAsync(d.rle2, d_syms, sizeof(uint16_t) * s, cudaMemcpyDeviceToDevice, st));
    set_int(d.s, s, st);
    set_int(d.n_in_use, n_in_use, st);
    BZ_CUDA(cudaMemsetAsync(d.freq, 0, sizeof(int32_t) * kMaxAlpha, st));
    k_histogram<<<std::min((s + 255) / 256, 296), 256, 0, st>>>(d.rle2, s, d.freq);
    BZ_LAUNCH_CHECK();
    stage_huffman(d, st);
    const int nsel = (s + 49) / 50;
    std::vector<uint8_t> hl(kMaxGroups * kMaxAlpha);
    std::vector<int32_t> hc(kMaxGroups * kMaxAlpha);
    int ng = 0;
    BZ_CUDA(cudaMemcpyAsync(hl.data(), d.len, hl.size(), cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(hc.data(), d.code, hc.size() * 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(selectors, d.sel, nsel, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(&ng, d.n_groups, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    const int alpha = n_in_use + 2;
    for (int t = 0; t < kMaxGroups; t++)
      for (int v = 0; v < alpha; v++) {
        len[t * kMaxAlpha + v] = hl[t * kMaxAlpha + v];
        if (t < ng) code[t * kMaxAlpha + v] = hc[t * kMaxAlpha + v];
      }
    *n_groups = ng;
    if (n_selectors) *n_selectors = nsel;
  });
}

int bz2g_huffman_encode(const uint16_t *d_syms, int s, const uint8_t *len, const int32_t *code,
                        const uint8_t *d_selectors, int n_selectors, int n_groups,
                        uint32_t *d_words, int64_t *bits, void *stream) {
  return guard([&] {
    BZ_REQUIRE(s > 0 && d_syms && len && code && d_selectors && d_words && bits, kErrArg,
               "bad arguments");
    BZ_REQUIRE(n_groups >= 1 && n_groups <= kMaxGroups, kErrArg, "n_groups outside [1, 6]");
    BZ_REQUIRE(n_selectors >= (s + 49) / 50, kErrArg, "too few selectors for s symbols");
    cudaStream_t st = S(stream);
    OneBlock ob(s, st);
    const SlabDev &d = ob.d();
    BZ_CUDA(cudaMemcpyAsync(d.rle2, d_syms, sizeof(uint16_t) * s, cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d.sel, d_selectors, (s + 49) / 50, cudaMemcpyDeviceToDevice, st));
    std::vector<uint8_t> hl(len, len + kMaxGroups * kMaxAlpha);
    std::vector<int32_t> hc(code, code + kMaxGroups * kMaxAlpha);
    BZ_CUDA(cudaMemcpyAsync(d.len, hl.data(), hl.size(), cudaMemcpyHostToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d.code, hc.data(), hc.size() * 4, cudaMemcpyHostToDevice, st));
    set_int(d.s, s, st);
    set_int(d.n_sel, (s + 49) / 50, st);
    set_int(d.n_groups, n_groups, st);
    stage_sizes_payload_only(d, st);
    int64_t total = 0;
    BZ_CUDA(cudaMemcpyAsync(&total, d.pay_bits, 8, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    BZ_CUDA(cudaMemsetAsync(d_words, 0, sizeof(uint32_t) * ((total + 31) / 32), st));
    launch_pack_words(d, d_words, st);
    BZ_CUDA(cudaStreamSynchronize(st));
    *bits = total;
  });
}

int bz2g_count_frequencies(const uint16_t *d_syms, int s, int32_t *d_freqs, void *stream) {
  return guard([&] {
    BZ_REQUIRE(s >= 0 && d_freqs, kErrArg, "bad arguments");
    if (s == 0) return;
    cudaStream_t st = S(stream);
    k_histogram<<<std::min((s + 255) / 256, 296), 256, 0, st>>>(d_syms, s, d_freqs);
    BZ_LAUNCH_CHECK();
    BZ_CUDA(cudaStreamSynchronize(st));
  });
}

}  // extern "C"

// ----------------------------------------------------- learned table selector
namespace {
// Error word of the training kernels, per device.
int *train_err() {
  static std::mutex mu;
  static std::map<int, int *> words;
  int dev = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  int *&w = words[dev];
  if (!w) {
    BZ_CUDA(cudaMalloc((void **)&w, 64));
    BZ_CUDA(cudaMemset(w, 0, 64));
  }
  return w;
}

mlp::Batch batch_views(int B, const void *X, const float *inv, const uint8_t *labels, void *work,
                       float *stats) {
  mlp::Batch b{};
  b.B = B;
  b.X = static_cast<const __nv_bfloat16 *>(X);
  b.inv = inv;
  b.labels = labels;
  uint8_t *p = static_cast<uint8_t *>(work);
  const size_t hb = align_up((int64_t)B * mlp::kHid * 2, 256);
  b.H1 = reinterpret_cast<__nv_bfloat16 *>(p);
  b.H2 = reinterpret_cast<__nv_bfloat16 *>(p + hb);
  b.dZ2 = reinterpret_cast<__nv_bfloat16 *>(p + 2 * hb);
  b.dZ1 = reinterpret_cast<__nv_bfloat16 *>(p + 3 * hb);
  b.Z3 = reinterpret_cast<float *>(p + 4 * hb);
  b.dZ3 = reinterpret_cast<__nv_bfloat16 *>(p + 4 * hb + align_up((int64_t)B * 64, 256));
  b.stats = stats;
  return b;
}
}  // namespace

extern "C" {

int bz2g_selector_load(const float *params, size_t count) {
  return guard([&] {
    BZ_REQUIRE(params && count == (size_t)mlp::kParams, kErrArg,
               "selector parameters: expected BZ2G_SELECTOR_PARAMS floats");
    int dev = 0;
    BZ_CUDA(cudaGetDevice(&dev));
    float *d = nullptr;
    uint8_t *packed = nullptr;
    BZ_CUDA(cudaMalloc((void **)&d, sizeof(float) * mlp::kParams));
    BZ_CUDA(cudaMemcpy(d, params, sizeof(float) * mlp::kParams, cudaMemcpyHostToDevice));
    BZ_CUDA(cudaMalloc((void **)&packed, mlp::kPackedBytes));
    mlp::pack(d, packed, 0);
    BZ_CUDA(cudaDeviceSynchronize());
    BZ_CUDA(cudaFree(d));
    std::lock_guard<std::mutex> g(g_sel_mu);
    uint8_t *&slot = g_sel_packed[dev];
    if (slot) BZ_CUDA(cudaFree(slot));
    slot = packed;
  });
}

int bz2g_set_selector(int mode) {
  return guard([&] {
    BZ_REQUIRE(mode >= 0 && mode <= 2, kErrArg, "selector mode must be 0, 1 or 2");
    std::lock_guard<std::mutex> g(g_sel_mu);
    g_sel_mode = mode;
  });
}

int bz2g_get_selector(void) {
  std::lock_guard<std::mutex> g(g_sel_mu);
  return g_sel_mode;
}

int bz2g_selector_logits(const uint16_t *d_syms, int s, const float *d_params, float *d_logits,
                         uint8_t *d_sel, void *stream) {
  return guard([&] {
    BZ_REQUIRE(s > 0 && d_syms && d_params && d_logits && d_sel, kErrArg, "bad arguments");
    cudaStream_t st = S(stream);
    OneBlock ob(s, st);
    const SlabDev &d = ob.d();
    const int nsel = (s + kGroupSize - 1) / kGroupSize;
    BZ_CUDA(cudaMemcpyAsync(d.rle2, d_syms, sizeof(uint16_t) * s, cudaMemcpyDeviceToDevice, st));
    set_int(d.s, s, st);
    set_int(d.n_sel, nsel, st);
    set_int(d.n_groups, kMaxGroups, st);
    set_int(d.learned, 1, st);
    BZ_CUDA(cudaMemsetAsync(d.rfreq, 0, sizeof(int32_t) * kMaxGroups * kMaxAlpha, st));
    float *raw = nullptr;
    BZ_CUDA(cudaMallocAsync((void **)&raw, sizeof(float) * 8 * kGroupTile * d.n_group_tiles, st));
    uint8_t *packed = pack_params(d_params, st);
    mlp::launch_select(d, packed, raw, nullptr, nullptr, st);
    BZ_CUDA(cudaMemcpy2DAsync(d_logits, 6 * sizeof(float), raw, 8 * sizeof(float),
                              6 * sizeof(float), nsel, cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d_sel, d.sel, nsel, cudaMemcpyDeviceToDevice, st));
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.err, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaFreeAsync(packed, st));
    BZ_CUDA(cudaFreeAsync(raw, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    BZ_REQUIRE(d.h_flags[0] == 0, kErrInternal, "selector kernel: a tensor-core wait timed out");
  });
}

int bz2g_selector_wait_check(const uint16_t *d_syms, int s, const float *d_params,
                             uint64_t wait_limit_ns, int withhold_weights, void *stream) {
  return guard([&] {
    BZ_REQUIRE(s > 0 && d_syms && d_params, kErrArg, "bad arguments");
    BZ_REQUIRE(wait_limit_ns > 0, kErrArg, "wait limit must be positive");
    cudaStream_t st = S(stream);
    OneBlock ob(s, st);
    const SlabDev &d = ob.d();
    const int nsel = (s + kGroupSize - 1) / kGroupSize;
    BZ_CUDA(cudaMemcpyAsync(d.rle2, d_syms, sizeof(uint16_t) * s, cudaMemcpyDeviceToDevice, st));
    set_int(d.s, s, st);
    set_int(d.n_sel, nsel, st);
    set_int(d.n_groups, kMaxGroups, st);
    set_int(d.learned, 1, st);
    BZ_CUDA(cudaMemsetAsync(d.rfreq, 0, sizeof(int32_t) * kMaxGroups * kMaxAlpha, st));
    BZ_CUDA(cudaMemsetAsync(d.err, 0, sizeof(int32_t), st));
    uint8_t *packed = pack_params(d_params, st);
    mlp::launch_select(d, packed, nullptr, nullptr, nullptr, st, wait_limit_ns,
                       withhold_weights ? 1 : 0);
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.err, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaFreeAsync(packed, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    BZ_REQUIRE(d.h_flags[0] == 0, kErrTimeout,
               "selector kernel: a bounded wait ran out (error word " +
                   std::to_string(d.h_flags[0]) + ")");
  });
}

int bz2g_huffman_build_learned(const uint16_t *d_syms, int s, int n_in_use, const float *d_params,
                               uint8_t *len, int32_t *code, uint8_t *selectors,
                               uint8_t *mlp_selectors, int *n_selectors, int *n_groups,
                               void *stream) {
  return guard([&] {
    BZ_REQUIRE(s > 0 && d_syms && d_params && len && code && selectors && n_groups, kErrArg,
               "bad arguments");
    BZ_REQUIRE(n_in_use >= 0 && n_in_use <= 256, kErrArg, "n_in_use outside [0, 256]");
    cudaStream_t st = S(stream);
    OneBlock ob(s, st);
    const SlabDev &d = ob.d();
    const int nsel = (s + kGroupSize - 1) / kGroupSize;
    BZ_CUDA(cudaMemcpyAsync(d.rle2, d_syms, sizeof(uint16_t) * s, cudaMemcpyDeviceToDevice, st));
    set_int(d.s, s, st);
    set_int(d.n_in_use, n_in_use, st);
    BZ_CUDA(cudaMemsetAsync(d.freq, 0, sizeof(int32_t) * kMaxAlpha, st));
    k_histogram<<<std::min((s + 255) / 256, 296), 256, 0, st>>>(d.rle2, s, d.freq);
    BZ_LAUNCH_CHECK();
    uint8_t *packed = pack_params(d_params, st);
    uint8_t *msel = nullptr;
    BZ_CUDA(cudaMallocAsync((void **)&msel, nsel, st));
    BZ_CUDA(cudaMemsetAsync(msel, 0, nsel, st));
    stage_huffman(d, st, packed, kIters, msel, nsel);
    std::vector<uint8_t> hl(kMaxGroups * kMaxAlpha);
    std::vector<int32_t> hc(kMaxGroups * kMaxAlpha);
    int ng = 0;
    BZ_CUDA(cudaMemcpyAsync(hl.data(), d.len, hl.size(), cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(hc.data(), d.code, hc.size() * 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(selectors, d.sel, nsel, cudaMemcpyDeviceToHost, st));
    if (mlp_selectors)
      BZ_CUDA(cudaMemcpyAsync(mlp_selectors, msel, nsel, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(&ng, d.n_groups, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.err, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaFreeAsync(packed, st));
    BZ_CUDA(cudaFreeAsync(msel, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    BZ_REQUIRE(d.h_flags[0] == 0, kErrInternal, "selector kernel: a tensor-core wait timed out");
    const int alpha = n_in_use + 2;
    for (int t = 0; t < kMaxGroups; t++)
      for (int v = 0; v < alpha; v++) {
        len[t * kMaxAlpha + v] = hl[t * kMaxAlpha + v];
        if (t < ng) code[t * kMaxAlpha + v] = hc[t * kMaxAlpha + v];
      }
    *n_groups = ng;
    if (n_selectors) *n_selectors = nsel;
  });
}

int bz2g_selector_dataset(int count, const uint8_t *const *d_inputs, const size_t *sizes,
                          const int *levels, uint16_t *d_group_syms, uint8_t *d_labels,
                          int64_t cap, int64_t *n_groups) {
  return guard([&] {
    BZ_REQUIRE(count >= 0 && (count == 0 || (d_inputs && sizes && levels)) && n_groups &&
                   cap >= 0 && (cap == 0 || (d_group_syms && d_labels)),
               kErrArg, "bad arguments");
    std::vector<Compressor::Item> items(count);
    int64_t maxb = 1;
    size_t bound = 64;
    for (int i = 0; i < count; i++) {
      const int lvl = std::min(std::max(levels[i], 1), 9);
      items[i] = {d_inputs[i], (int64_t)sizes[i], lvl, 100000 * lvl};
      maxb = std::max<int64_t>(maxb, 100000 * lvl);
      bound += stream_bound((int64_t)sizes[i], ((int64_t)sizes[i] + 100000 * lvl - 1) / (100000 * lvl));
    }
    // one worker: slabs in a fixed order, so the groups come in a fixed order
    CompressorConfig cfg;
    cfg.slab_blocks = g_slab;
    cfg.workers = 1;
    cfg.max_block_bytes = std::max<int64_t>(maxb, 900000);
    int64_t *ctl = nullptr;
    BZ_CUDA(cudaMalloc((void **)&ctl, sizeof(int64_t) * (1 + cfg.slab_blocks)));
    BZ_CUDA(cudaMemset(ctl, 0, sizeof(int64_t) * (1 + cfg.slab_blocks)));
    mlp::SelectorTap tap{d_group_syms, d_labels, cap, ctl, ctl + 1};
    cfg.tap = &tap;
    try {
      Compressor c(cfg);
      ByteSink sink;
      sink.reserve(bound);
      std::vector<size_t> offs;
      c.compress_batch(items.data(), count, true, sink, offs, nullptr);
      BZ_CUDA(cudaMemcpy(n_groups, ctl, sizeof(int64_t), cudaMemcpyDeviceToHost));
    } catch (...) {
      cudaFree(ctl);
      throw;
    }
    BZ_CUDA(cudaFree(ctl));
  });
}

int bz2g_mlp_features(const uint16_t *d_group_syms, int64_t G, void *d_X, float *d_inv,
                      void *stream) {
  return guard([&] {
    BZ_REQUIRE(G >= 0 && (G == 0 || (d_group_syms && d_X && d_inv)), kErrArg, "bad arguments");
    mlp::features(d_group_syms, G, static_cast<__nv_bfloat16 *>(d_X), d_inv, S(stream));
  });
}

size_t bz2g_mlp_work_bytes(int B) {
  if (B <= 0) return 0;
  return (size_t)(4 * align_up((int64_t)B * mlp::kHid * 2, 256) + align_up((int64_t)B * 64, 256) +
                  align_up((int64_t)B * 32, 256));
}

int bz2g_mlp_grads(const void *d_p16, const float *d_params, int B, const void *d_X,
                   const float *d_inv, const uint8_t *d_labels, void *d_work, float *d_grad,
                   float *d_stats, void *stream) {
  return guard([&] {
    BZ_REQUIRE(B > 0 && B % 128 == 0, kErrArg, "batch must be a positive multiple of 128");
    BZ_REQUIRE(d_p16 && d_params && d_X && d_inv && d_labels && d_work && d_grad && d_stats,
               kErrArg, "null device pointer");
    mlp::Batch b = batch_views(B, d_X, d_inv, d_labels, d_work, d_stats);
    mlp::grads(static_cast<const __nv_bfloat16 *>(d_p16), d_params, b, d_grad, train_err(),
               S(stream));
  });
}

int bz2g_mlp_forward(const void *d_p16, const float *d_params, int B, const void *d_X,
                     const float *d_inv, void *d_work, float *d_logits, void *stream) {
  return guard([&] {
    BZ_REQUIRE(B > 0 && B % 128 == 0, kErrArg, "batch must be a positive multiple of 128");
    BZ_REQUIRE(d_p16 && d_params && d_X && d_inv && d_work && d_logits, kErrArg,
               "null device pointer");
    mlp::Batch b = batch_views(B, d_X, d_inv, nullptr, d_work, nullptr);
    b.Z3 = d_logits;
    mlp::forward(static_cast<const __nv_bfloat16 *>(d_p16), d_params, b, train_err(), S(stream));
  });
}

int bz2g_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, void *d_p16,
                  float lr, float beta1, float beta2, float eps, int step, void *stream) {
  return guard([&] {
    BZ_REQUIRE(d_params && d_grad && d_m && d_v && d_p16 && step >= 1, kErrArg, "bad arguments");
    mlp::adam(d_params, d_grad, d_m, d_v, static_cast<__nv_bfloat16 *>(d_p16), lr, beta1, beta2,
              eps, step, S(stream));
  });
}

int bz2g_mlp_to_bf16(const float *d_params, void *d_p16, void *stream) {
  return guard([&] {
    BZ_REQUIRE(d_params && d_p16, kErrArg, "null device pointer");
    mlp::to_bf16(d_params, static_cast<__nv_bfloat16 *>(d_p16), S(stream));
  });
}

int bz2g_mlp_status(void *stream) {
  return guard([&] {
    int *w = train_err();
    int h = 0;
    cudaStream_t st = S(stream);
    BZ_CUDA(cudaMemcpyAsync(&h, w, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    if (h) BZ_CUDA(cudaMemset(w, 0, 4));
    BZ_REQUIRE(h == 0, kErrInternal,
               "training kernels: a tensor-core wait timed out (error word " +
                   std::to_string(h) + ")");
  });
}

}  // extern "C"

// ------------------------------------------------ one stream over several GPUs
extern "C" {

size_t bz2g_part_bound(size_t n, int block_bytes) {
  if (block_bytes <= 0) block_bytes = 900000;
  size_t nb = (n + block_bytes - 1) / block_bytes;
  return stream_bound((int64_t)n, (int64_t)nb) + 16;
}

int bz2g_compress_part(const uint8_t *in, size_t n, int block_bytes, int on_device,
                       uint8_t *d_part, size_t cap, int64_t *bits, uint32_t *crc_fold,
                       int *nblocks) {
  return guard([&] {
    BZ_REQUIRE(d_part && bits && crc_fold && nblocks, kErrArg, "null output pointer");
    BZ_REQUIRE(block_bytes > 0 && block_bytes <= (1 << 24), kErrArg,
               "block_bytes must be in (0, 16 MiB]");
    BZ_REQUIRE(n == 0 || in != nullptr, kErrArg, "null input");
    BZ_REQUIRE((uintptr_t)d_part % 4 == 0, kErrArg, "part buffer must be 4-byte aligned");
    const int64_t nb = ((int64_t)n + block_bytes - 1) / block_bytes;
    std::vector<const uint8_t *> ptrs(nb);
    std::vector<int> lens(nb);
    for (int64_t b = 0; b < nb; b++) {
      ptrs[b] = in + b * (int64_t)block_bytes;
      lens[b] = (int)std::min<int64_t>(block_bytes, (int64_t)n - b * (int64_t)block_bytes);
    }
    ByteSink sink(d_part, cap);
    BZ_REQUIRE(sink.device, kErrArg, "the part buffer must be device memory");
    Compressor &c = engine_for(std::max<int64_t>(block_bytes, 1));
    set_format(c);
    g_last_stats = StageTimes();
    int64_t b = 0;
    uint32_t f = 0;
    if (nb > 0) c.compress_part(ptrs.data(), lens.data(), (int)nb, on_device != 0, sink, &b, &f,
                                &g_last_stats);
    // zero the bytes after the part up to a 4-byte boundary (splice reads words)
    const size_t used = (size_t)((b + 7) / 8);
    const size_t end = (used + 3) / 4 * 4;
    BZ_REQUIRE(end <= cap, kErrTooLarge, "part buffer too small");
    if (end > used) BZ_CUDA(cudaMemset(d_part + used, 0, end - used));
    BZ_CUDA(cudaDeviceSynchronize());
    *bits = b;
    *crc_fold = f;
    *nblocks = (int)nb;
  });
}

int bz2g_assemble(int nparts, const uint8_t *const *d_parts, const int64_t *bits,
                  const uint32_t *crc_folds, const int *nblocks, int level, uint8_t *out,
                  size_t cap, size_t *out_len) {
  return guard([&] {
    BZ_REQUIRE(nparts >= 0 && out && out_len && (nparts == 0 || (d_parts && bits && crc_folds &&
                                                                   nblocks)),
               kErrArg, "bad arguments");
    const int lvl = std::min(std::max(level, 1), 9);
    int64_t total = 32;
    uint32_t crc = 0;
    // splice in segments of 2^20 source words, one CTA each
    const int64_t seg_bits = int64_t(1) << 25;
    std::vector<int64_t> src, dst, nb;
    for (int r = 0; r < nparts; r++) {
      BZ_REQUIRE(bits[r] >= 0 && (bits[r] == 0 || d_parts[r]), kErrArg, "bad part");
      BZ_REQUIRE((uintptr_t)d_parts[r] % 4 == 0, kErrArg, "parts must be 4-byte aligned");
      for (int64_t o = 0; o < bits[r]; o += seg_bits) {
        src.push_back((int64_t)(uintptr_t)(d_parts[r] + o / 8));
        dst.push_back(total + o);
        nb.push_back(std::min<int64_t>(seg_bits, bits[r] - o));
      }
      total += bits[r];
      const int k = ((nblocks[r] % 32) + 32) % 32;
      crc = (k ? ((crc << k) | (crc >> (32 - k))) : crc) ^ crc_folds[r];
    }
    const size_t stream_bytes = (size_t)((total + 80 + 7) / 8);
    BZ_REQUIRE(stream_bytes <= cap, kErrTooLarge, "output buffer too small");
    const int64_t words = (total + 31) / 32 + 1;
    const int ns = (int)src.size();
    cudaStream_t st = 0;
    uint32_t *d_out = nullptr;
    int64_t *d_meta = nullptr;
    BZ_CUDA(cudaMallocAsync((void **)&d_out, sizeof(uint32_t) * words, st));
    BZ_CUDA(cudaMallocAsync((void **)&d_meta, sizeof(int64_t) * 3 * std::max(ns, 1), st));
    BZ_CUDA(cudaMemsetAsync(d_out, 0, sizeof(uint32_t) * words, st));
    if (ns > 0) {
      BZ_CUDA(cudaMemcpyAsync(d_meta, src.data(), 8 * ns, cudaMemcpyHostToDevice, st));
      BZ_CUDA(cudaMemcpyAsync(d_meta + ns, dst.data(), 8 * ns, cudaMemcpyHostToDevice, st));
      BZ_CUDA(cudaMemcpyAsync(d_meta + 2 * ns, nb.data(), 8 * ns, cudaMemcpyHostToDevice, st));
      launch_splice(d_meta, d_meta + ns, d_meta + 2 * ns, ns, d_out, st);
    }
    const size_t body = (size_t)((total + 7) / 8);
    BZ_CUDA(cudaMemcpyAsync(out, d_out, body, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaFreeAsync(d_meta, st));
    BZ_CUDA(cudaFreeAsync(d_out, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    out[0] = 'B';
    out[1] = 'Z';
    out[2] = 'h';
    out[3] = (uint8_t)('0' + lvl);
    ByteSink view(out, cap);
    view.size = body;
    put_eos(view, 0, total, crc);
    *out_len = view.size;
  });
}

}  // extern "C"

// ------------------------------------------------------------- file streams
extern "C" int bz2g_compress_file(const char *in_path, const char *out_path, int level,
                                  int group_blocks) {
  return guard([&] {
    const int group = group_blocks > 0 ? group_blocks : kGroupBlocks;
    std::unique_ptr<BZFileInputStream> in;
    if (in_path) {
      FILE *probe = std::fopen(in_path, "rb");
      BZ_REQUIRE(probe != nullptr, kErrArg, std::string("cannot open input file: ") + in_path);
      std::fclose(probe);
      in.reset(new BZFileInputStream(2 * group, 900000, std::string(in_path)));
    } else {
      in.reset(new BZFileInputStream(2 * group, 900000));
    }
    FILE *out = out_path ? std::fopen(out_path, "wb") : stdout;
    BZ_REQUIRE(out != nullptr, kErrArg, std::string("cannot open output file: ") + out_path);
    bool write_failed = false;
    try {
      Compressor &c = default_engine(900000);
      StreamWriter w(c, level, [&](const uint8_t *p, size_t k) {
        if (!write_failed && std::fwrite(p, 1, k, out) != k) write_failed = true;
      });
      compress_input_stream(*in, w, group);
    } catch (...) {
      if (out_path) std::fclose(out);
      throw;
    }
    if (std::fflush(out) != 0) write_failed = true;
    if (out_path && std::fclose(out) != 0) write_failed = true;
    BZ_REQUIRE(!in->failed(), kErrArg, "reading the input failed");
    BZ_REQUIRE(!write_failed, kErrArg, "writing the output failed");
  });
}

