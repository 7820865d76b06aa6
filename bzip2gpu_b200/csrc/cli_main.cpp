// bzip2gpu command line tool (reference: src/main.cpp:20-60).  Blocks are
// 900,000 raw bytes for every level, as in the reference (its input stream
// always uses 900000-byte buffers); the level only sets the header digit.
// Input is read ahead into a ring of pinned chunks while earlier groups of
// blocks compress, and output is written as each group finishes.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "bz2g.h"
#include "cli.h"

int main(int argc, char **argv) {
  CliOptions opt = parse_args(argc, argv);
  const bool timing = std::getenv("BZ2G_TIMING") != nullptr;
  auto t0 = std::chrono::steady_clock::now();
  int rc = 0;
  if (opt.input_files.empty()) {
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
