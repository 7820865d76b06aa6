// Drop-in C++ API (include/compression.h, io.h, cli.h, crc32.h) over the
// C-ABI.  Errors print and exit(EXIT_FAILURE), as the reference's
// CUDA_ERROR_CHECK does (reference include/utils.h:3-12).
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>

#include <condition_variable>
#include <cstring>
#include <deque>
#include <fstream>
#include <iostream>
#include <mutex>
#include <thread>
#include <vector>

#include "bz2g.h"
#include "cli.h"
#include "compression.h"
#include "compressor.h"
#include "crc32.h"
#include "engine.h"
#include "io.h"
#include "stream.h"

namespace {

void die_on(int status, const char *what) {
  if (status != BZ2G_OK) {
    fprintf(stderr, "%s failed: %s\n", what, bz2g_last_error());
    exit(EXIT_FAILURE);
  }
}

void die_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    fprintf(stderr, "%s failed: %s (%s)\n", what, cudaGetErrorName(e), cudaGetErrorString(e));
    exit(EXIT_FAILURE);
  }
}

}  // namespace

// ------------------------------------------------------------ compression.h

int rle1_compress(const uint8_t *in, int in_len, uint8_t *&out, cudaStream_t stream) {
  if (in_len == 0) return 0;
  die_cuda(cudaMallocAsync((void **)&out, bz2g_rle1_bound((size_t)in_len), stream),
           "rle1_compress: cudaMallocAsync");
  int m = 0;
  die_on(bz2g_rle1(in, in_len, out, &m, stream), "rle1_compress");
  return m;
}

void rle2_compress(const uint8_t *in, int in_len, uint16_t *out, uint32_t *out_len,
                   int table_size, cudaStream_t stream) {
  die_on(bz2g_rle2(in, in_len, table_size, out, out_len, stream), "rle2_compress");
}

int make_symbols_table(const uint8_t *d_in, int d_in_len, uint8_t *&symbols_table,
                       cudaStream_t stream) {
  uint8_t tbl[256];
  int count = 0;
  die_on(bz2g_symbols_table(d_in, d_in_len, tbl, &count, stream), "make_symbols_table");
  symbols_table = new uint8_t[count];
  std::memcpy(symbols_table, tbl, count);
  return count;
}

int fmtf(const uint8_t *in_original, const int *in_suffix_array, int in_len, uint8_t *&out,
         int &orig_ptr, bool *present_symbols, cudaStream_t stream) {
  if (in_len == 0) return 0;
  die_cuda(cudaMallocAsync((void **)&out, in_len, stream), "fmtf: cudaMallocAsync");
  uint8_t pres[256];
  int n_in_use = 0;
  die_on(bz2g_mtf(in_original, in_suffix_array, in_len, out, &orig_ptr, pres, &n_in_use, stream),
         "fmtf");
  if (present_symbols)
    for (int i = 0; i < 256; i++) present_symbols[i] = pres[i] != 0;
  return n_in_use;
}

int huffman_build_trees(uint16_t *device_data_in, int data_in_len, int alphabet_size,
                        uint8_t len[max_n_groups][max_alphabet_size],
                        int32_t code[max_n_groups][max_alphabet_size], uint8_t *&selectors,
                        int &n_groups, cudaStream_t stream) {
  const int nsel = (data_in_len + 49) / 50;
  selectors = new uint8_t[nsel > 0 ? nsel : 1];
  int got = 0;
  die_on(bz2g_huffman_build(device_data_in, data_in_len, alphabet_size, &len[0][0], &code[0][0],
                            selectors, &got, &n_groups, stream),
         "huffman_build_trees");
  return got;
}

void fbwt(const uint8_t *in, int in_len, int *&out, cudaStream_t stream) {
  if (in_len == 0) return;
  die_cuda(cudaMallocAsync((void **)&out, sizeof(int) * (size_t)in_len, stream),
           "fbwt: cudaMallocAsync");
  die_on(bz2g_bwt(in, in_len, out, stream), "fbwt");
}

int huffman_encode(uint16_t *dev_data_in, int data_in_len, int alphabet_size,
                   uint32_t *&dev_encoded_data, uint8_t len[max_n_groups][max_alphabet_size],
                   int32_t code[max_n_groups][max_alphabet_size], uint8_t *dev_selectors,
                   int32_t num_selectors, int n_groups, cudaStream_t stream) {
  (void)alphabet_size;  // the reference ignores it too
  const size_t words = ((size_t)data_in_len * 17 + 31) / 32 + 1;
  die_cuda(cudaMalloc((void **)&dev_encoded_data, words * sizeof(uint32_t)),
           "huffman_encode: cudaMalloc");
  int64_t bits = 0;
  die_on(bz2g_huffman_encode(dev_data_in, data_in_len, &len[0][0], &code[0][0], dev_selectors,
                             num_selectors, n_groups, dev_encoded_data, &bits, stream),
         "huffman_encode");
  return (int)bits;
}

__global__ void count_frequencies(uint16_t *data_in, int data_len, int *freqs) {
  int idx = blockDim.x * blockIdx.x + threadIdx.x;
  if (idx < data_len) atomicAdd(&freqs[data_in[idx]], 1);
}

// Streams the input through the GPU in groups of blocks (stream.h): the
// stream's pinned chunks are reused, at most kGroupBlocks are held at a time,
// and the output grows as groups finish.
void bzip2_gpu_compress(BZFileInputStream &in_stream, int n, std::vector<uint8_t> &out) {
  try {
    bz2g::Compressor &c = bz2g::default_engine(std::max(in_stream.buffer_size(), 1));
    bz2g::StreamWriter w(c, n, [&](const uint8_t *p, size_t k) { out.insert(out.end(), p, p + k); });
    bz2g::compress_input_stream(in_stream, w);
  } catch (const std::exception &e) {
    fprintf(stderr, "bzip2_gpu_compress failed: %s\n", e.what());
    exit(EXIT_FAILURE);
  }
}

namespace bz2g {
void compress_input_stream(BZFileInputStream &in, StreamWriter &w, int group_blocks) {
  std::vector<uint8_t *> bufs;
  std::vector<const uint8_t *> cbufs;
  std::vector<int> lens;
  auto flush = [&] {
    w.add(cbufs.data(), lens.data(), (int)lens.size(), false);
    for (uint8_t *b : bufs) in.release(b);
    bufs.clear();
    cbufs.clear();
    lens.clear();
  };
  uint8_t *p;
  int idx, len;
  while ((len = in.fetch_pooled(p, idx)) >= 0) {
    if (len == 0) {
      in.release(p);
      continue;
    }
    bufs.push_back(p);
    cbufs.push_back(p);
    lens.push_back(len);
    if ((int)lens.size() >= group_blocks) flush();
  }
  if (!lens.empty()) flush();
  w.finish();
}
}  // namespace bz2g

// --------------------------------------------------------------------- io.h

struct BZFileInputStream::Impl {
  std::istream *in = nullptr;
  std::ifstream file;
  int n_buffers, buffer_size;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::pair<uint8_t *, int>> q;
  std::vector<uint8_t *> free_bufs;  // pinned buffers given back by release()
  bool closed = false, failed = false, stop = false;
  int next_idx = 0;
  std::thread th;

  void reader() {
    for (;;) {
      uint8_t *buf = nullptr;
      {
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&] { return (int)q.size() < n_buffers || stop; });
        if (stop) break;
        if (!free_bufs.empty()) {
          buf = free_bufs.back();
          free_bufs.pop_back();
        }
      }
      if (!buf && cudaMallocHost((void **)&buf, buffer_size) != cudaSuccess) {
        std::lock_guard<std::mutex> g(mu);
        failed = true;
        break;
      }
      in->read(reinterpret_cast<char *>(buf), buffer_size);
      int got = (int)in->gcount();
      bool bad = in->bad();
      std::lock_guard<std::mutex> g(mu);
      if (got > 0) q.emplace_back(buf, got);
      else free_bufs.push_back(buf);
      if (bad) failed = true;
      if (got < buffer_size || bad) break;
      cv.notify_all();
    }
    std::lock_guard<std::mutex> g(mu);
    closed = true;
    cv.notify_all();
  }
};

static BZFileInputStream::Impl *make_impl(int n_buffers, int buffer_size) {
  auto *im = new BZFileInputStream::Impl();
  im->n_buffers = n_buffers > 0 ? n_buffers : 1;
  im->buffer_size = buffer_size > 0 ? buffer_size : 1;
  return im;
}

BZFileInputStream::BZFileInputStream(int n_buffers, int buffer_size)
    : impl_(make_impl(n_buffers, buffer_size)) {
  impl_->in = &std::cin;
  impl_->th = std::thread(&Impl::reader, impl_);
}

BZFileInputStream::BZFileInputStream(int n_buffers, int buffer_size, std::string filename)
    : impl_(make_impl(n_buffers, buffer_size)) {
  impl_->file.open(filename, std::ios::in | std::ios::binary);
  if (!impl_->file) {
    fprintf(stderr, "cannot open input file: %s\n", filename.c_str());
    impl_->failed = true;
    impl_->closed = true;
    return;
  }
  impl_->in = &impl_->file;
  impl_->th = std::thread(&Impl::reader, impl_);
}

BZFileInputStream::~BZFileInputStream() {
  {
    std::lock_guard<std::mutex> g(impl_->mu);
    impl_->stop = true;
    impl_->cv.notify_all();
  }
  if (impl_->th.joinable()) impl_->th.join();
  for (auto &e : impl_->q) cudaFreeHost(e.first);
  for (uint8_t *b : impl_->free_bufs) cudaFreeHost(b);
  delete impl_;
}

int BZFileInputStream::fetch(uint8_t *&result, int &chunk_idx) {
  std::unique_lock<std::mutex> g(impl_->mu);
  impl_->cv.wait(g, [&] { return !impl_->q.empty() || impl_->closed; });
  if (impl_->q.empty()) return -1;
  auto e = impl_->q.front();
  impl_->q.pop_front();
  result = e.first;
  chunk_idx = impl_->next_idx++;
  impl_->cv.notify_all();
  return e.second;
}

int BZFileInputStream::fetch_pooled(uint8_t *&result, int &chunk_idx) {
  return fetch(result, chunk_idx);
}

void BZFileInputStream::release(uint8_t *chunk) {
  if (!chunk) return;
  std::lock_guard<std::mutex> g(impl_->mu);
  impl_->free_bufs.push_back(chunk);
  impl_->cv.notify_all();
}

bool BZFileInputStream::failed() const {
  std::lock_guard<std::mutex> g(impl_->mu);
  return impl_->failed;
}

int BZFileInputStream::buffer_size() const { return impl_->buffer_size; }

// ------------------------------------------------------------------ crc32.h

void crc32_init() {}

uint32_t bzip2_crc32(const uint8_t *data, size_t length) {
  if (length == 0) return 0;
  uint8_t *d = nullptr;
  die_cuda(cudaMalloc((void **)&d, length), "bzip2_crc32: cudaMalloc");
  die_cuda(cudaMemcpy(d, data, length, cudaMemcpyHostToDevice), "bzip2_crc32: copy");
  uint32_t crc = 0;
  die_on(bz2g_crc32(d, length, &crc, nullptr), "bzip2_crc32");
  cudaFree(d);
  return crc;
}

// -------------------------------------------------------------------- cli.h

static void show_help() {
  printf(
      "bzip2gpu (B200): bzip2 compression on the GPU\n"
      "   usage: bzip2gpu [flags and input files in any order]\n"
      "\n"
      "   -h --help           print this message\n"
      "   -z --compress       force compression\n"
      "   -c --stdout         output to standard out\n"
      "   -1 .. -9            set the block size digit (100k .. 900k)\n"
      "   --fast              alias for -1\n"
      "   --best              alias for -9\n"
      "\n"
      "   With no file names, compresses standard input to standard output.\n"
      "   Short flags combine: -z -4 is the same as -z4.\n");
}

CliOptions parse_args(int argc, char **argv) {
  CliOptions opt;
  static struct option longs[] = {{"help", no_argument, 0, 'h'},
                                  {"compress", no_argument, 0, 'z'},
                                  {"stdout", no_argument, 0, 'c'},
                                  {"fast", no_argument, 0, '1'},
                                  {"best", no_argument, 0, '9'},
                                  {0, 0, 0, 0}};
  optind = 1;
  for (;;) {
    int c = getopt_long(argc, argv, ":hzc123456789", longs, nullptr);
    if (c == -1) break;
    if (c >= '1' && c <= '9') {
      opt.block_size = c - '0';
      continue;
    }
    switch (c) {
      case 'z':
        opt.compress = true;
        break;
      case 'c':
        opt.stdout_output = true;
        break;
      case 'h':
        show_help();
        exit(EXIT_SUCCESS);
      case ':':
        fprintf(stderr, "Missing argument\n");
        exit(EXIT_FAILURE);
      default:
        if (optopt) fprintf(stderr, "UNKNOWN OPTION: -%c\n", optopt);
        else fprintf(stderr, "UNKNOWN OPTION: %s\n", argv[optind - 1]);
        show_help();
        exit(EXIT_FAILURE);
    }
  }
  while (optind < argc) opt.input_files.push_back(argv[optind++]);
  return opt;
}
