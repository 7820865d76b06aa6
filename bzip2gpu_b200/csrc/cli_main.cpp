// bzip2gpu command line tool (reference: src/main.cpp:20-60).  Blocks are
// 900,000 raw bytes for every level, as in the reference (its input stream
// always uses 900000-byte buffers); the level only sets the header digit.
// Input is read ahead into a ring of pinned chunks while earlier groups of
// blocks compress, and output is written as each group finishes.
//
// With BZ2G_BZIP2_FORMAT=1 in the environment, streams use bzip2 1.0.8's
// block format instead (libbz2's block split and 255-byte runs, so every
// level gives a stream any bzip2 decoder accepts, byte-identical to libbz2's):
// each input is read whole, as that split walks the entire input.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "bz2g.h"
#include "cli.h"

namespace {

// Whole input (path, or standard input when null); false if it cannot be read.
bool read_all(const char *path, std::vector<uint8_t> &data) {
  FILE *f = path ? std::fopen(path, "rb") : stdin;
  if (!f) return false;
  uint8_t buf[1 << 16];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) data.insert(data.end(), buf, buf + k);
  const bool ok = !std::ferror(f);
  if (path) std::fclose(f);
  return ok;
}

// One input in bzip2 1.0.8's block format; false (message set) on failure.
bool compress_bzip2_format(const char *in_path, const char *out_path, int level) {
  std::vector<uint8_t> data;
  if (!read_all(in_path, data)) {
    std::cerr << "bzip2gpu: cannot read " << (in_path ? in_path : "standard input") << std::endl;
    return false;
  }
  uint8_t *out = nullptr;
  size_t len = 0;
  if (bz2g_compress(data.data(), data.size(), level, BZ2G_BZIP2_BLOCKS, &out, &len) != BZ2G_OK) {
    std::cerr << "bzip2gpu: " << bz2g_last_error() << std::endl;
    return false;
  }
  FILE *f = out_path ? std::fopen(out_path, "wb") : stdout;
  bool ok = f && std::fwrite(out, 1, len, f) == len;
  if (f && out_path) ok = std::fclose(f) == 0 && ok;
  if (!out_path) std::fflush(stdout);
  bz2g_free(out);
  if (!ok) std::cerr << "bzip2gpu: cannot write " << (out_path ? out_path : "standard output")
                     << std::endl;
  return ok;
}

}  // namespace

int main(int argc, char **argv) {
  CliOptions opt = parse_args(argc, argv);
  const bool timing = std::getenv("BZ2G_TIMING") != nullptr;
  const char *fmt = std::getenv("BZ2G_BZIP2_FORMAT");
  const bool bzip2_format = fmt != nullptr && fmt[0] == '1';
  auto t0 = std::chrono::steady_clock::now();
  int rc = 0;
  if (bzip2_format) {
    if (opt.input_files.empty()) {
      rc = compress_bzip2_format(nullptr, nullptr, opt.block_size) ? 0 : 1;
    } else {
      for (const auto &file : opt.input_files) {
        const std::string out = opt.stdout_output ? std::string() : file + ".bz2";
        if (!compress_bzip2_format(file.c_str(), opt.stdout_output ? nullptr : out.c_str(),
                                   opt.block_size))
          rc = 1;
      }
    }
  } else if (opt.input_files.empty()) {
    if (bz2g_compress_file(nullptr, nullptr, opt.block_size, 0) != BZ2G_OK) {
      std::cerr << "bzip2gpu: " << bz2g_last_error() << std::endl;
      rc = 1;
    }
  } else {
    for (const auto &file : opt.input_files) {
      const std::string out = opt.stdout_output ? std::string() : file + ".bz2";
      if (bz2g_compress_file(file.c_str(), opt.stdout_output ? nullptr : out.c_str(),
                             opt.block_size, 0) != BZ2G_OK) {
        std::cerr << "bzip2gpu: " << file << ": " << bz2g_last_error() << std::endl;
        rc = 1;
      }
    }
  }
  std::cout.flush();
  if (timing) {
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                    .count();
    std::cerr << "All: " << ms << "\n";
  }
  return rc;
}
